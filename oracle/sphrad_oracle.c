/*
 * sphrad_oracle.c -- CPU oracle for the sphradiometer cross-power path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker used by tests/, by smoke() and by
 * the CPU-baseline leg of bench.py.  The product library never links or
 * calls this file.  Everything here is a plain FP64 restatement of the
 * reference's algorithms (cannon-zz/sphradiometer); each function cites
 * the reference lines it follows.  Third-party numerics that the
 * reference takes from GSL and FFTW (associated Legendre functions,
 * Gauss-Legendre tables, Wigner 3-j symbols, FFTs) are restated from their
 * published algorithms, so agreement with GSL/FFTW themselves is pinned
 * only through the reference's own test tolerances.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "sphrad_oracle.h"
#include "ref_shims/bfgs2.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------ */
/* index math: sh_series.h:172-227                                     */
/* ------------------------------------------------------------------ */

size_t orc_moffset(unsigned l_max, int m)
{
	const long L = (long) l_max + 1;
	const long x = (long) m * (m - 1);
	if(m >= 0)
		return (size_t) (L * m - x / 2);
	return (size_t) (L * (L + m) + x / 2);
}

size_t orc_lmoffset(unsigned l_max, unsigned l, int m)
{
	return orc_moffset(l_max, m) + l - abs(m);
}

size_t orc_length(unsigned l_max, int polar)
{
	return polar ? (size_t) l_max + 1 : ((size_t) l_max + 1) * ((size_t) l_max + 1);
}

/* ------------------------------------------------------------------ */
/* Legendre functions (GSL sphPlm convention, used at                  */
/* sh_series_trans.c:68,93,627,715,836,847)                            */
/* ------------------------------------------------------------------ */

/* P~_l^m(x) = (-1)^m sqrt((2l+1)/(4pi) (l-m)!/(l+m)!) P_l^m(x), by the
 * standard three-term recurrence in l started from the sectoral value,
 * whose prefactor is formed in log space so that it underflows quietly. */
void orc_sphPlm_array(int l_max, int m, double x, double *out)
{
	double lnpre = 0.5 * log((2.0 * m + 1.0) / (4.0 * M_PI));
	for(int i = 1; i <= m; i++)
		lnpre += 0.5 * log((2.0 * i - 1.0) / (2.0 * i));
	double pmm = (m > 0) ? exp(lnpre + 0.5 * m * log1p(-x * x)) : exp(lnpre);
	if(m & 1)
		pmm = -pmm;
	if(l_max < m)
		return;
	out[0] = pmm;
	if(l_max == m)
		return;
	double p1 = x * sqrt(2.0 * m + 3.0) * pmm;
	out[1] = p1;
	double p0 = pmm;
	for(int l = m + 2; l <= l_max; l++) {
		const double a = sqrt((2.0 * l + 1.0) * (2.0 * l - 1.0) / ((double) (l - m) * (l + m)));
		const double b = sqrt((2.0 * l + 1.0) * (l + m - 1.0) * (l - m - 1.0) / ((2.0 * l - 3.0) * (l - m) * (l + m)));
		const double p = a * x * p1 - b * p0;
		out[l - m] = p;
		p0 = p1;
		p1 = p;
	}
}

/* sh_series_trans.c:65-69 */
double complex orc_Y(unsigned l, int m, double theta, double phi)
{
	const int am = abs(m);
	double *P = malloc((l - am + 1) * sizeof(*P));
	orc_sphPlm_array(l, am, cos(theta), P);
	double v = P[l - am];
	free(P);
	const double sign = (m < 0 && (am & 1)) ? -1.0 : 1.0;
	return sign * (cos(m * phi) + I * sin(m * phi)) * v;
}

/* ------------------------------------------------------------------ */
/* Gauss-Legendre quadrature (sh_series_trans.c:149-196)               */
/* ------------------------------------------------------------------ */

/* Newton iteration on P_n for the roots in (0, 1), mirrored to (-1, 0).
 * Output is ordered by decreasing x, i.e. increasing theta, as the
 * reference's pixels_from_l_max() reverses GSL's table. */
void orc_gl_nodes(int n, double *x, double *w)
{
	const int half = (n + 1) / 2;
	for(int i = 0; i < half; i++) {
		double z = cos(M_PI * (i + 0.75) / (n + 0.5));
		double pp = 0.0;
		for(int it = 0; it < 100; it++) {
			double p0 = 1.0, p1 = z;
			for(int k = 2; k <= n; k++) {
				double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
				p0 = p1;
				p1 = p2;
			}
			if(n == 1) {
				p1 = z;
				p0 = 1.0;
			}
			pp = n * (z * p1 - p0) / (z * z - 1.0);
			double dz = p1 / pp;
			z -= dz;
			if(fabs(dz) < 1e-16)
				break;
		}
		/* recompute derivative at the converged root */
		{
			double p0 = 1.0, p1 = z;
			for(int k = 2; k <= n; k++) {
				double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
				p0 = p1;
				p1 = p2;
			}
			if(n == 1) {
				p1 = z;
				p0 = 1.0;
			}
			pp = n * (z * p1 - p0) / (z * z - 1.0);
		}
		x[i] = z;
		x[n - 1 - i] = -z;
		w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
	}
	if(n & 1)
		x[n / 2] = 0.0;
}

/* ------------------------------------------------------------------ */
/* DFT (FFTW's unnormalised convention: sign -1 forward, +1 backward)  */
/* ------------------------------------------------------------------ */

static void fft_radix2(double complex *a, int n, int sign)
{
	for(int i = 1, j = 0; i < n; i++) {
		int bit = n >> 1;
		for(; j & bit; bit >>= 1)
			j ^= bit;
		j ^= bit;
		if(i < j) {
			double complex t = a[i];
			a[i] = a[j];
			a[j] = t;
		}
	}
	for(int len = 2; len <= n; len <<= 1) {
		for(int i = 0; i < n; i += len)
			for(int k = 0; k < len / 2; k++) {
				const double ang = sign * 2.0 * M_PI * k / len;
				const double complex w = cos(ang) + I * sin(ang);
				double complex u = a[i + k], v = a[i + k + len / 2] * w;
				a[i + k] = u + v;
				a[i + k + len / 2] = u - v;
			}
	}
}

void orc_dft(double complex *data, int n, int sign)
{
	if(n <= 1)
		return;
	if((n & (n - 1)) == 0) {
		fft_radix2(data, n, sign);
		return;
	}
	/* direct sum with exactly-indexed twiddles */
	double complex *tw = malloc(n * sizeof(*tw));
	double complex *out = malloc(n * sizeof(*out));
	for(int k = 0; k < n; k++) {
		const double ang = sign * 2.0 * M_PI * k / n;
		tw[k] = cos(ang) + I * sin(ang);
	}
	for(int k = 0; k < n; k++) {
		double complex s = 0.0;
		long idx = 0;
		for(int j = 0; j < n; j++) {
			s += data[j] * tw[idx];
			idx += k;
			if(idx >= n)
				idx -= n;
		}
		out[k] = s;
	}
	memcpy(data, out, n * sizeof(*out));
	free(out);
	free(tw);
}

/* ------------------------------------------------------------------ */
/* series arithmetic (sh_series.c)                                     */
/* ------------------------------------------------------------------ */

/* sh_series_assign() semantics (sh_series.c:123-184), out of place:
 * copies the coefficients both series hold and zeroes the rest of dst. */
void orc_assign(double complex *dst, unsigned dst_l, int dst_polar, const double complex *src, unsigned src_l, int src_polar)
{
	const size_t n = orc_length(dst_l, dst_polar);
	double complex *tmp = calloc(n, sizeof(*tmp));
	const unsigned l_min = dst_l < src_l ? dst_l : src_l;
	const int m_max = (dst_polar || src_polar) ? 0 : (int) l_min;
	for(int m = -m_max; m <= m_max; m++)
		for(unsigned l = abs(m); l <= l_min; l++)
			tmp[orc_lmoffset(dst_l, l, m)] = src[orc_lmoffset(src_l, l, m)];
	memcpy(dst, tmp, n * sizeof(*tmp));
	free(tmp);
}

/* sh_series.c:441-475 */
void orc_conj(double complex *a, unsigned l_max, int polar)
{
	const int m_max = polar ? 0 : (int) l_max;
	for(unsigned l = 0; l <= l_max; l++)
		a[orc_lmoffset(l_max, l, 0)] = conj(a[orc_lmoffset(l_max, l, 0)]);
	for(int m = 1; m <= m_max; m++)
		for(unsigned l = m; l <= l_max; l++) {
			const double complex ap = a[orc_lmoffset(l_max, l, m)];
			const double complex an = a[orc_lmoffset(l_max, l, -m)];
			const double s = (m & 1) ? -1.0 : 1.0;
			a[orc_lmoffset(l_max, l, m)] = s * conj(an);
			a[orc_lmoffset(l_max, l, -m)] = s * conj(ap);
		}
}

/* sh_series_rotation.c:600-625 */
void orc_rotate_z(double complex *a, unsigned l_max, int polar, double phi)
{
	if(polar)
		return;
	for(int m = -(int) l_max; m <= (int) l_max; m++) {
		const double complex f = cos(-m * phi) + I * sin(-m * phi);
		for(unsigned l = abs(m); l <= l_max; l++)
			a[orc_lmoffset(l_max, l, m)] *= f;
	}
}

/* sh_series_trans.c:257-291, summed in the same order */
double complex orc_eval(const double complex *a, unsigned l_max, int polar, double theta, double phi)
{
	double *P = malloc((l_max + 1) * sizeof(*P));
	const int m_max = polar ? 0 : (int) l_max;
	const double x = cos(theta);
	double complex val = 0.0;
	for(int m = 0; m <= m_max; m++) {
		orc_sphPlm_array(l_max, m, x, P);
		const double complex e = cos(m * phi) + I * sin(m * phi);
		double complex xp = 0.0, xm = 0.0;
		for(unsigned l = m; l <= l_max; l++) {
			const double complex y = e * P[l - m];
			xp += a[orc_lmoffset(l_max, l, m)] * y;
			if(m)
				xm += a[orc_lmoffset(l_max, l, -m)] * conj(y);
		}
		val += xp + ((m & 1) ? -xm : xm);
	}
	free(P);
	return val;
}

/* sh_series.c:645-676 (plain sum; the reference sorts by magnitude
 * first, which only changes rounding) */
double complex orc_dot(const double complex *a, const double complex *b, unsigned l_max, int polar)
{
	const size_t n = orc_length(l_max, polar);
	double complex s = 0.0;
	for(size_t i = n; i-- > 0;)
		s += a[i] * conj(b[i]);
	return s;
}

/* ------------------------------------------------------------------ */
/* transforms on the Gauss-Legendre mesh (sh_series_trans.c:575-871)   */
/* ------------------------------------------------------------------ */

void orc_to_mesh(const double complex *a, unsigned l_max, int polar, double complex *mesh)
{
	const int nt = 2 * (l_max + 1), np = nt;
	const int m_max = polar ? 0 : (int) l_max;
	double *x = malloc(nt * sizeof(*x)), *w = malloc(nt * sizeof(*w));
	double *P = malloc((l_max + 1) * sizeof(*P));
	orc_gl_nodes(nt, x, w);
	memset(mesh, 0, (size_t) nt * np * sizeof(*mesh));
	for(int i = 0; i < nt; i++) {
		double complex *F = mesh + (size_t) i * np;
		for(int m = 0; m <= m_max; m++) {
			orc_sphPlm_array(l_max, m, x[i], P);
			double complex xp = 0.0, xm = 0.0;
			for(unsigned l = m; l <= l_max; l++) {
				xp += a[orc_lmoffset(l_max, l, m)] * P[l - m];
				if(m)
					xm += a[orc_lmoffset(l_max, l, -m)] * P[l - m];
			}
			F[m] = xp;
			if(m)
				F[np - m] = (m & 1) ? -xm : xm;
		}
		orc_dft(F, np, +1);
	}
	free(P);
	free(w);
	free(x);
}

void orc_from_mesh(double complex *a, unsigned l_max, int polar, const double complex *mesh)
{
	const int nt = 2 * (l_max + 1), np = nt;
	const int m_max = polar ? 0 : (int) l_max;
	double *x = malloc(nt * sizeof(*x)), *w = malloc(nt * sizeof(*w));
	double *P = malloc((size_t) nt * (l_max + 1) * sizeof(*P));
	double complex *F = malloc((size_t) nt * np * sizeof(*F));
	orc_gl_nodes(nt, x, w);
	memcpy(F, mesh, (size_t) nt * np * sizeof(*F));
	for(int i = 0; i < nt; i++) {
		orc_dft(F + (size_t) i * np, np, -1);
		const double wt = w[i] * (2.0 * M_PI / np);
		for(int j = 0; j < np; j++)
			F[(size_t) i * np + j] *= wt;
	}
	for(int m = 0; m <= m_max; m++) {
		for(int i = 0; i < nt; i++)
			orc_sphPlm_array(l_max, m, x[i], P + (size_t) i * (l_max + 1));
		for(unsigned l = m; l <= l_max; l++) {
			double complex c = 0.0, cn = 0.0;
			for(int i = 0; i < nt; i++) {
				const double p = P[(size_t) i * (l_max + 1) + (l - m)];
				c += F[(size_t) i * np + m] * p;
				if(m)
					cn += F[(size_t) i * np + np - m] * p;
			}
			a[orc_lmoffset(l_max, l, m)] = c;
			if(m)
				a[orc_lmoffset(l_max, l, -m)] = ((m & 1) ? -1.0 : 1.0) * cn;
		}
	}
	free(F);
	free(P);
	free(w);
	free(x);
}

/* sh_series_trans.c:885-899 */
void orc_impulse(double complex *a, unsigned l_max, double theta, double phi)
{
	for(int m = -(int) l_max; m <= (int) l_max; m++)
		for(unsigned l = abs(m); l <= l_max; l++)
			a[orc_lmoffset(l_max, l, m)] = conj(orc_Y(l, m, theta, phi));
}

/* ------------------------------------------------------------------ */
/* rotations (sh_series_rotation.c)                                    */
/* ------------------------------------------------------------------ */

/* sh_series_rotation.c:104-153: Rz(alpha) Ry(beta) Rz(gamma) */
void orc_euler_rotation_matrix(double gamma, double beta, double alpha, double *R)
{
	const double ca = cos(alpha), sa = sin(alpha);
	const double cb = cos(beta), sb = sin(beta);
	const double cg = cos(gamma), sg = sin(gamma);
	R[0] = ca * cb * cg - sa * sg;
	R[1] = -ca * cb * sg - sa * cg;
	R[2] = ca * sb;
	R[3] = sa * cb * cg + ca * sg;
	R[4] = -sa * cb * sg + ca * cg;
	R[5] = sa * sb;
	R[6] = -sb * cg;
	R[7] = sb * sg;
	R[8] = cb;
}

size_t orc_rot_offset(unsigned l)
{
	/* sum_{k=1}^{l-1} (2k+1)^2 */
	size_t s = 0;
	for(unsigned k = 1; k < l; k++)
		s += (size_t) (2 * k + 1) * (2 * k + 1);
	return s;
}

size_t orc_rot_plan_len(unsigned l_max)
{
	return orc_rot_offset(l_max + 1);
}

#define DEL(D, l, m, mp) (D)[(size_t) (2 * (l) + 1) * ((mp) + (l)) + ((m) + (l))]

/* Choi, Ivanic, Gordon & Ruedenberg recursion coefficients
 * (sh_series_rotation.c:316-341) */
static double ca_(int l, int m, int mp) { return sqrt((double) (l + m) * (l - m) / ((double) (l + mp) * (l - mp))); }
static double cb_(int l, int m, int mp) { return sqrt((double) (l + m) * (l + m - 1) / (2.0 * (l + mp) * (l - mp))); }
static double cc_(int l, int m, int mp) { return sqrt(2.0 * (l + m) * (l - m) / ((double) (l + mp) * (l + mp - 1))); }
static double cd_(int l, int m, int mp) { return sqrt((double) (l + m) * (l + m - 1) / ((double) (l + mp) * (l + mp - 1))); }

/* sh_series_rotation.c:287-310 (l = 1) and :346-369 (l > 1) */
void orc_rotation_plan(unsigned l_max, const double *R, double complex *Dall)
{
	enum { x = 0, y = 1, z = 2 };
	if(l_max < 1)
		return;
	double complex *D1 = Dall;
	const double s2 = sqrt(2.0);
	DEL(D1, 1, -1, -1) = (R[3 * y + y] + R[3 * x + x] - I * (R[3 * x + y] - R[3 * y + x])) / 2;
	DEL(D1, 1, -1, 0) = (R[3 * z + x] - I * R[3 * z + y]) / s2;
	DEL(D1, 1, -1, +1) = (R[3 * y + y] - R[3 * x + x] + I * (R[3 * x + y] + R[3 * y + x])) / 2;
	DEL(D1, 1, 0, -1) = (R[3 * x + z] + I * R[3 * y + z]) / s2;
	DEL(D1, 1, 0, 0) = R[3 * z + z];
	DEL(D1, 1, 0, +1) = (-R[3 * x + z] + I * R[3 * y + z]) / s2;
	DEL(D1, 1, +1, -1) = (R[3 * y + y] - R[3 * x + x] - I * (R[3 * x + y] + R[3 * y + x])) / 2;
	DEL(D1, 1, +1, 0) = (-R[3 * z + x] - I * R[3 * z + y]) / s2;
	DEL(D1, 1, +1, +1) = (R[3 * y + y] + R[3 * x + x] - I * (R[3 * y + x] - R[3 * x + y])) / 2;
	for(int l = 2; l <= (int) l_max; l++) {
		const double complex *Dp = Dall + orc_rot_offset(l - 1);
		double complex *D = Dall + orc_rot_offset(l);
		const int lp = l - 1;
		for(int m = -l; m <= l; m++) {
			for(int mp = -l + 1; mp <= l - 1; mp++) {
				double complex v = 0.0;
				if(abs(m) != l)
					v += ca_(l, m, mp) * DEL(D1, 1, 0, 0) * DEL(Dp, lp, m, mp);
				if(m > -l + 1)
					v += cb_(l, m, mp) * DEL(D1, 1, 1, 0) * DEL(Dp, lp, m - 1, mp);
				if(-m > -l + 1)
					v += cb_(l, -m, mp) * DEL(D1, 1, -1, 0) * DEL(Dp, lp, m + 1, mp);
				DEL(D, l, m, mp) = v;
			}
			{
				const int mp = -l;
				double complex v = 0.0;
				if(abs(m) != l)
					v += cc_(l, m, -mp) * DEL(D1, 1, 0, -1) * DEL(Dp, lp, m, mp + 1);
				if(m > -l + 1)
					v += cd_(l, m, -mp) * DEL(D1, 1, 1, -1) * DEL(Dp, lp, m - 1, mp + 1);
				if(-m > -l + 1)
					v += cd_(l, -m, -mp) * DEL(D1, 1, -1, -1) * DEL(Dp, lp, m + 1, mp + 1);
				DEL(D, l, m, mp) = v;
			}
			{
				const int mp = l;
				double complex v = 0.0;
				if(abs(m) != l)
					v += cc_(l, m, mp) * DEL(D1, 1, 0, 1) * DEL(Dp, lp, m, mp - 1);
				if(m > -l + 1)
					v += cd_(l, m, mp) * DEL(D1, 1, 1, 1) * DEL(Dp, lp, m - 1, mp - 1);
				if(-m > -l + 1)
					v += cd_(l, -m, mp) * DEL(D1, 1, -1, 1) * DEL(Dp, lp, m + 1, mp - 1);
				DEL(D, l, m, mp) = v;
			}
		}
	}
}

/* sh_series_rotation.c:546-589; result is a non-polar series of the
 * same l_max.  Returns -1 where the reference returns NULL. */
int orc_rotate(double complex *result, const double complex *series, unsigned l_max, int polar, const double complex *Dall)
{
	if(result == series)
		return -1;
	result[0] = series[0];
	for(int l = 1; l <= (int) l_max; l++) {
		const double complex *D = Dall + orc_rot_offset(l);
		for(int mp = -l; mp <= l; mp++) {
			double complex c;
			if(polar)
				c = DEL(D, l, 0, mp) * series[orc_lmoffset(l_max, l, 0)];
			else {
				c = 0.0;
				for(int m = -l; m <= l; m++)
					c += DEL(D, l, m, mp) * series[orc_lmoffset(l_max, l, m)];
			}
			result[orc_lmoffset(l_max, l, mp)] = c;
		}
	}
	return 0;
}

/* ------------------------------------------------------------------ */
/* Wigner 3-j symbols.  The reference calls GSL (sh_series_product.c:  */
/* 80-83).  Restated here with the Schulten-Gordon three-term          */
/* recursion in j1 (J. Math. Phys. 16, 1961 (1975)): recurse upward    */
/* from j1min and downward from j1max, join where the downward         */
/* solution stops growing, normalise by sum (2j1+1) f^2 = 1 and fix    */
/* the sign of the j1max value to (-1)^(j2-j3-m1).                     */
/* ------------------------------------------------------------------ */

static double sg_A(double j, double j2, double j3, double m1)
{
	const double v = (j * j - (j2 - j3) * (j2 - j3)) * ((j2 + j3 + 1) * (j2 + j3 + 1) - j * j) * (j * j - m1 * m1);
	return v > 0 ? sqrt(v) : 0.0;
}

static double sg_B(double j, double j2, double j3, double m1, double m2, double m3)
{
	return -(2 * j + 1) * (j2 * (j2 + 1) * m1 - j3 * (j3 + 1) * m1 - j * (j + 1) * (m3 - m2));
}

/* fills f[j1 - j1min]; returns the number of values (0 if none) */
static int wigner_3j_j1(int j2, int j3, int m2, int m3, int *j1min_out, double *f)
{
	const int m1 = -m2 - m3;
	if(abs(m2) > j2 || abs(m3) > j3)
		return 0;
	const int j1min = abs(j2 - j3) > abs(m1) ? abs(j2 - j3) : abs(m1);
	const int j1max = j2 + j3;
	if(j1max < j1min)
		return 0;
	const int n = j1max - j1min + 1;
	*j1min_out = j1min;
	const double sgn = ((j2 - j3 - m1) & 1) ? -1.0 : 1.0;
	if(n == 1) {
		f[0] = sgn / sqrt(2.0 * j1min + 1);
		return 1;
	}
	/* downward from j1max */
	double *fb = f;
	fb[n - 1] = 1.0;
	/* jturn: lowest j1 taken from the downward pass.  The downward pass
	 * stops at the first j1 where it stops growing (the end of the
	 * upper classically forbidden region); below that the upward pass
	 * is the stable one.  A pass that grows all the way down (or any
	 * pass with j1min = 0, where the upward start is degenerate) is
	 * kept whole. */
	int jturn = j1min;
	{
		int j = j1max;
		double fnext = 0.0; /* f(j + 1) */
		while(j > j1min) {
			const double Aj = sg_A(j, j2, j3, m1);
			const double Aj1 = sg_A(j + 1, j2, j3, m1);
			const double v = -(sg_B(j, j2, j3, m1, m2, m3) * fb[j - j1min] + j * Aj1 * fnext) / ((j + 1) * Aj);
			fnext = fb[j - j1min];
			fb[j - 1 - j1min] = v;
			j--;
			if(fabs(v) > 1e100) {
				for(int k = j - j1min; k < n; k++)
					fb[k] *= 1e-100;
				fnext *= 1e-100;
			}
			if(j1min > 0 && fabs(fb[j - j1min]) < fabs(fb[j + 1 - j1min])) {
				jturn = j + 1;
				break;
			}
		}
	}
	if(jturn > j1min) {
		/* upward from j1min up to jturn + 2 (capped), then match */
		const int jtop = (jturn + 2 < j1max) ? jturn + 2 : j1max;
		double *ff = malloc((jtop - j1min + 1) * sizeof(*ff));
		ff[0] = 1.0;
		double fprev = 0.0;
		for(int j = j1min; j < jtop; j++) {
			const double Aj = sg_A(j, j2, j3, m1);
			const double Aj1 = sg_A(j + 1, j2, j3, m1);
			const double v = -(sg_B(j, j2, j3, m1, m2, m3) * ff[j - j1min] + (j + 1) * Aj * fprev) / (j * Aj1);
			fprev = ff[j - j1min];
			ff[j + 1 - j1min] = v;
			if(fabs(v) > 1e100) {
				for(int k = 0; k <= j + 1 - j1min; k++)
					ff[k] *= 1e-100;
				fprev *= 1e-100;
			}
		}
		double num = 0.0, den = 0.0;
		for(int j = jturn; j <= jtop; j++) {
			num += ff[j - j1min] * fb[j - j1min];
			den += ff[j - j1min] * ff[j - j1min];
		}
		const double scale = num / den;
		for(int j = j1min; j < jturn; j++)
			f[j - j1min] = ff[j - j1min] * scale;
		free(ff);
	}
	double norm = 0.0;
	for(int k = 0; k < n; k++)
		norm += (2.0 * (j1min + k) + 1) * f[k] * f[k];
	norm = 1.0 / sqrt(norm);
	if((f[n - 1] < 0) != (sgn < 0))
		norm = -norm;
	for(int k = 0; k < n; k++)
		f[k] *= norm;
	return n;
}

double orc_wigner_3j(int j1, int j2, int j3, int m1, int m2, int m3)
{
	if(m1 + m2 + m3 != 0 || abs(m1) > j1 || abs(m2) > j2 || abs(m3) > j3)
		return 0.0;
	if(j1 < abs(j2 - j3) || j1 > j2 + j3)
		return 0.0;
	double *f = malloc((j2 + j3 + 2) * sizeof(*f));
	int j1min = 0;
	const int n = wigner_3j_j1(j2, j3, m2, m3, &j1min, f);
	double v = 0.0;
	if(n > 0 && j1 >= j1min && j1 < j1min + n)
		v = f[j1 - j1min];
	free(f);
	return v;
}

/* ------------------------------------------------------------------ */
/* products (sh_series_product.c)                                      */
/* ------------------------------------------------------------------ */

/* enumeration of sh_series_product.c:123-162; with factor == NULL only
 * counts.  Ops come out grouped by dest l, m ascending; the reference
 * then sorts them by (dest, a, b) offsets, which only reorders the
 * summation. */
static long product_plan_impl(int Dl, int Dp, int Al, int Ap, int Bl, int Bp, double *factor, int *d_off, int *a_off, int *b_off)
{
	long n = 0;
	for(int dl = 0; dl <= Dl; dl++) {
		const int dm_max = (Dp || (Ap && Bp)) ? 0 : dl;
		for(int dm = -dm_max; dm <= dm_max; dm++) {
			const int al_min = dl > Bl ? dl - Bl : 0;
			const int al_max = Al < dl + Bl ? Al : dl + Bl;
			for(int al = al_min; al <= al_max; al++) {
				const int bl_max = Bl < dl + al ? Bl : dl + al;
				int bl_min = abs(dl - al);
				bl_min += (al + bl_min + dl) & 1;
				for(int bl = bl_min; bl <= bl_max; bl += 2) {
					int am_min = -(al < bl - dm ? al : bl - dm);
					int am_max = al < bl + dm ? al : bl + dm;
					if(Ap) {
						if(am_min > 0 || am_max < 0)
							continue;
						am_min = am_max = 0;
					}
					double g0 = 0.0;
					if(factor)
						g0 = sqrt((2.0 * dl + 1) * (2.0 * al + 1) * (2.0 * bl + 1) / (4 * M_PI)) * orc_wigner_3j(al, bl, dl, 0, 0, 0);
					for(int am = am_min; am <= am_max; am++) {
						const int bm = dm - am;
						if(Bp && bm != 0)
							continue;
						if(factor) {
							factor[n] = ((dm & 1) ? -1.0 : 1.0) * g0 * orc_wigner_3j(al, bl, dl, am, bm, -dm);
							d_off[n] = (int) orc_lmoffset(Dl, dl, dm);
							a_off[n] = (int) orc_lmoffset(Al, al, am);
							b_off[n] = (int) orc_lmoffset(Bl, bl, bm);
						}
						n++;
					}
				}
			}
		}
	}
	return n;
}

long orc_product_plan_length(unsigned d_l, int d_polar, unsigned a_l, int a_polar, unsigned b_l, int b_polar)
{
	if(d_l > a_l + b_l)
		d_l = a_l + b_l;
	return product_plan_impl(d_l, d_polar, a_l, a_polar, b_l, b_polar, NULL, NULL, NULL, NULL);
}

long orc_product_plan(unsigned d_l, int d_polar, unsigned a_l, int a_polar, unsigned b_l, int b_polar, double *factor, int *d_off, int *a_off, int *b_off)
{
	if(d_l > a_l + b_l)
		d_l = a_l + b_l;
	return product_plan_impl(d_l, d_polar, a_l, a_polar, b_l, b_polar, factor, d_off, a_off, b_off);
}

/* sh_series_product.c:250-266.  Offsets index a dest of l_max d_l'
 * = min(d_l, a_l + b_l); this restatement takes the plan's own dest
 * l_max, so callers pass the truncated value. */
void orc_product_microcode(double complex *dest, unsigned d_l, int d_polar, const double complex *a, const double complex *b, long n_ops, const double *factor, const int *d_off, const int *a_off, const int *b_off)
{
	memset(dest, 0, orc_length(d_l, d_polar) * sizeof(*dest));
	for(long i = 0; i < n_ops; i++)
		dest[d_off[i]] += a[a_off[i]] * b[b_off[i]] * factor[i];
}

/* sh_series_product.c:269-329 */
void orc_product_pixel(double complex *dest, unsigned d_l, int d_polar, const double complex *a, unsigned a_l, int a_polar, const double complex *b, unsigned b_l, int b_polar)
{
	const unsigned L = a_l + b_l;
	const size_t nt = 2 * (L + 1);
	double complex *wa = malloc(orc_length(L, a_polar) * sizeof(*wa));
	double complex *wb = malloc(orc_length(L, b_polar) * sizeof(*wb));
	double complex *ma = malloc(nt * nt * sizeof(*ma));
	double complex *mb = malloc(nt * nt * sizeof(*mb));
	orc_assign(wa, L, a_polar, a, a_l, a_polar);
	orc_assign(wb, L, b_polar, b, b_l, b_polar);
	orc_to_mesh(wa, L, a_polar, ma);
	orc_to_mesh(wb, L, b_polar, mb);
	for(size_t i = 0; i < nt * nt; i++)
		ma[i] *= mb[i];
	const int p = a_polar && b_polar;
	double complex *wr = malloc(orc_length(L, p) * sizeof(*wr));
	orc_from_mesh(wr, L, p, ma);
	orc_assign(dest, d_l, d_polar, wr, L, p);
	free(wr);
	free(mb);
	free(ma);
	free(wb);
	free(wa);
}

/* ------------------------------------------------------------------ */
/* delay kernel (projection.c, correlator.c:55-65, 325-519)            */
/* ------------------------------------------------------------------ */

/* projection.c:56-66 */
int orc_projection_n_elements(double r, double delta_t)
{
	return 2 * (int) (60 + r / delta_t + 1) + 1;
}

/* projection.c:75-87 */
unsigned orc_projection_l_max(double r, double delta_t)
{
	const int l = M_PI * r / delta_t + 1;
	return l;
}

/* correlator.c:55-65 */
unsigned orc_power_l_max_naive(double d, double delta_t)
{
	return floor(M_PI / (2. * asin(delta_t / (2. * d))) + 1.);
}

/* projection.c:99-131 for a phase centre at r * z-hat: the polar
 * projection of the sinc delay taps.  taps[t * (a_l_max + 1) + l], with
 * tap t at delay k = t - (n_el - 1) / 2.  The reference samples the tap
 * on the full Gauss-Legendre mesh and keeps the m = 0 bin of its phi
 * transform (sh_series_trans.c:663-734); for a phase centre on the z
 * axis r.s = r cos(theta) exactly, the samples do not depend on phi and
 * that bin is nphi times the ring value, which is what is used here. */
void orc_projection_taps(double r, double delta_t, int n_el, unsigned a_l_max, double *taps)
{
	const int nt = 2 * (a_l_max + 1);
	double *x = malloc(nt * sizeof(*x)), *w = malloc(nt * sizeof(*w));
	double *P = malloc((size_t) nt * (a_l_max + 1) * sizeof(*P));
	orc_gl_nodes(nt, x, w);
	for(int i = 0; i < nt; i++)
		orc_sphPlm_array(a_l_max, 0, x[i], P + (size_t) i * (a_l_max + 1));
	for(int t = 0; t < n_el; t++) {
		const int k = t - (n_el - 1) / 2;
		double *out = taps + (size_t) t * (a_l_max + 1);
		memset(out, 0, (a_l_max + 1) * sizeof(*out));
		for(int i = 0; i < nt; i++) {
			const double pi_x = M_PI * (0 - k - r * cos(acos(x[i])) / delta_t);
			const double s = (pi_x == 0.0) ? 1.0 : sin(pi_x) / pi_x;
			const double f = 2.0 * M_PI * w[i] * s;
			const double *Pi = P + (size_t) i * (a_l_max + 1);
			for(unsigned l = 0; l <= a_l_max; l++)
				out[l] += f * Pi[l];
		}
	}
	free(P);
	free(w);
	free(x);
}

/* correlator.c:424-519 for a baseline of length d_len (seconds), keeping
 * the delay product up to l_max (the effect of correlator_plan_fd_set_l,
 * correlator.c:571-591).  D is n x (l_max + 1), polar.  The per-bin
 * product conj(A_i) B_i is evaluated with the quadrature of the
 * reference's pixel-domain product (sh_series_product.c:269-329): polar
 * factors are constant on each mesh ring, so the product reduces to a
 * Gauss-Legendre sum in cos(theta); 2 (a_l_max + 1) nodes integrate the
 * degree 2 a_l_max + l_max integrand exactly, as the reference's larger
 * mesh does.  Returns -1 on bad arguments. */
int orc_delay_product(double d_len, double delta_t, int n, unsigned l_max, double complex *D)
{
	const double r = d_len / 2;
	if(d_len <= 0 || delta_t <= 0 || n <= 0)
		return -1;
	const unsigned a_l = orc_projection_l_max(r, delta_t);
	const int n_el = orc_projection_n_elements(r, delta_t);
	unsigned p_l = orc_power_l_max_naive(d_len, delta_t);
	if(p_l > 2 * a_l)
		p_l = 2 * a_l;
	if(l_max > p_l)
		return -1;
	const int A = a_l + 1;
	double *ta = malloc((size_t) n_el * A * sizeof(*ta));
	double *tb = malloc((size_t) n_el * A * sizeof(*tb));
	orc_projection_taps(+r, delta_t, n_el, a_l, ta);
	orc_projection_taps(-r, delta_t, n_el, a_l, tb);
	/* zero-pad the tap axis to n and transform (correlator.c:446-451,
	 * sh_series_array.c:125-171, 528-539) */
	double complex *tw = malloc(n * sizeof(*tw));
	for(int k = 0; k < n; k++)
		tw[k] = cos(-2.0 * M_PI * k / n) + I * sin(-2.0 * M_PI * k / n);
	const int nt = 2 * A;
	/* Legendre table up to max(a_l_max, l_max) */
	const int LP = (int) (a_l > l_max ? a_l : l_max) + 1;
	double *x = malloc(nt * sizeof(*x)), *w = malloc(nt * sizeof(*w));
	double *P = malloc((size_t) nt * LP * sizeof(*P));
	orc_gl_nodes(nt, x, w);
	for(int i = 0; i < nt; i++)
		orc_sphPlm_array(LP - 1, 0, x[i], P + (size_t) i * LP);
	const int n_tap = n_el < n ? n_el : n;
#pragma omp parallel for schedule(dynamic, 16)
	for(int f = 0; f < n; f++) {
		double complex *Af = malloc(A * sizeof(*Af));
		double complex *Bf = malloc(A * sizeof(*Bf));
		for(int l = 0; l < A; l++)
			Af[l] = Bf[l] = 0.0;
		long idx = 0;
		for(int t = 0; t < n_tap; t++) {
			const double complex e = tw[idx];
			const double *pa = ta + (size_t) t * A, *pb = tb + (size_t) t * A;
			for(int l = 0; l < A; l++) {
				Af[l] += pa[l] * e;
				Bf[l] += pb[l] * e;
			}
			idx += f;
			idx %= n;
		}
		/* conj(A) (correlator.c:484-486) times B, projected to l <= l_max */
		double complex *out = D + (size_t) ((n - f) % n) * (l_max + 1);
		for(unsigned l = 0; l <= l_max; l++)
			out[l] = 0.0;
		for(int i = 0; i < nt; i++) {
			const double *Pi = P + (size_t) i * LP;
			double complex u = 0.0, v = 0.0;
			for(int l = 0; l < A; l++) {
				u += conj(Af[l]) * Pi[l];
				v += Bf[l] * Pi[l];
			}
			const double complex h = 2.0 * M_PI * w[i] * u * v;
			for(unsigned l = 0; l <= l_max; l++)
				out[l] += h * Pi[l];
		}
		/* one factor of 1/n (correlator.c:492) */
		for(unsigned l = 0; l <= l_max; l++)
			out[l] *= 1.0 / n;
		free(Bf);
		free(Af);
	}
	free(P);
	free(w);
	free(x);
	free(tw);
	free(tb);
	free(ta);
	return 0;
}

/* ------------------------------------------------------------------ */
/* correlator (correlator.c:681-711, 993-1010)                         */
/* ------------------------------------------------------------------ */

int orc_baseline_integrate_power_fd(const double complex *a, const double complex *b, int n, const double complex *D, unsigned l_max, const double complex *Rot, double complex *power_2d)
{
	const int S = l_max + 1;
	double complex *p1 = calloc(S, sizeof(*p1));
	for(int k = 0; k < n; k++) {
		const double complex v = b[k] * conj(a[k]);
		const double complex *d = D + (size_t) k * S;
		for(int l = 0; l < S; l++)
			p1[l] += d[l] * v;
	}
	for(int l = 0; l < S; l++)
		p1[l] *= 1.0 / n;
	int rc = orc_rotate(power_2d, p1, l_max, 1, Rot);
	free(p1);
	return rc;
}

int orc_network_integrate_power_fd(int n_det, const double complex *const *fseries, int n, const double complex *const *D, unsigned l_max, const double complex *const *Rot, double complex *sky)
{
	const size_t len = orc_length(l_max, 0);
	const int nb = n_det * (n_det - 1) / 2;
	double complex *p2 = malloc(len * sizeof(*p2));
	memset(sky, 0, len * sizeof(*sky));
	int k = 0;
	for(int i = 1; i < n_det; i++)
		for(int j = 0; j < i; j++, k++) {
			if(orc_baseline_integrate_power_fd(fseries[i], fseries[j], n, D[k], l_max, Rot[k], p2)) {
				free(p2);
				return -1;
			}
			for(size_t q = 0; q < len; q++)
				sky[q] += (1.0 / nb) * p2[q];
		}
	free(p2);
	return 0;
}

/* correlator.c:325-400 and 648-673: the time-domain correlator of a
 * baseline of length d_len (seconds), as the reference runs it.  The
 * projections are the polar taps of +-d_len/2 z-hat; for each of the
 * n - 2 transient samples the two samples' series are formed
 * (sh_series_array_dot, sh_series_array.c:407-426), multiplied with the
 * Gaunt microcode (sh_series_product.c:250-266) into degree
 * min(l_max, 2 a_l_max) and added, times the window, into power_1d,
 * which is then rotated with Rot.  l_max is the plan's power l_max.
 * Returns -1 when n < 2 transient. */
int orc_baseline_integrate_power_td(const double *a, const double *b, const double *window, int n, double d_len, double delta_t, unsigned l_max,
				    const double complex *Rot, double complex *power_2d)
{
	const double r = d_len / 2;
	const unsigned a_l = orc_projection_l_max(r, delta_t);
	const int n_el = orc_projection_n_elements(r, delta_t);
	const int transient = (n_el - 1) / 2;
	const int T = n - 2 * transient;
	if(T < 0 || delta_t <= 0)
		return -1;
	const int A = a_l + 1;
	const unsigned dl = l_max < 2 * a_l ? l_max : 2 * a_l;
	double *ta = malloc((size_t) n_el * A * sizeof(*ta));
	double *tb = malloc((size_t) n_el * A * sizeof(*tb));
	orc_projection_taps(+r, delta_t, n_el, a_l, ta);
	orc_projection_taps(-r, delta_t, n_el, a_l, tb);
	const long n_ops = orc_product_plan_length(dl, 1, a_l, 1, a_l, 1);
	double *f = malloc((n_ops ? n_ops : 1) * sizeof(*f));
	int *d_off = malloc((n_ops ? n_ops : 1) * sizeof(*d_off));
	int *a_off = malloc((n_ops ? n_ops : 1) * sizeof(*a_off));
	int *b_off = malloc((n_ops ? n_ops : 1) * sizeof(*b_off));
	orc_product_plan(dl, 1, a_l, 1, a_l, 1, f, d_off, a_off, b_off);
	double complex *sa = malloc(A * sizeof(*sa)), *sb = malloc(A * sizeof(*sb));
	double complex *prod = malloc((dl + 1) * sizeof(*prod));
	double complex *p1 = calloc(l_max + 1, sizeof(*p1));
	for(int t = 0; t < T; t++) {
		for(int l = 0; l < A; l++)
			sa[l] = sb[l] = 0.0;
		for(int e = 0; e < n_el; e++) {
			const double va = a[t + e], vb = b[t + e];
			for(int l = 0; l < A; l++) {
				sa[l] += ta[(size_t) e * A + l] * va;
				sb[l] += tb[(size_t) e * A + l] * vb;
			}
		}
		orc_product_microcode(prod, dl, 1, sa, sb, n_ops, f, d_off, a_off, b_off);
		for(unsigned l = 0; l <= dl; l++)
			p1[l] += window[t] * prod[l];
	}
	const int rc = orc_rotate(power_2d, p1, l_max, 1, Rot);
	free(p1);
	free(prod);
	free(sb);
	free(sa);
	free(b_off);
	free(a_off);
	free(d_off);
	free(f);
	free(tb);
	free(ta);
	return rc;
}

/* instrument.c:90-100 */
void orc_vector_direction(const double *v, double *theta, double *phi)
{
	*theta = atan2(sqrt(v[0] * v[0] + v[1] * v[1]), v[2]);
	*phi = atan2(v[1], v[0]);
	if(*phi < 0)
		*phi += 2. * M_PI;
}

void orc_render_grid(const double complex *a, unsigned l_max, int polar, int ntheta, int nphi, double *grid)
{
#pragma omp parallel for
	for(int j = 0; j < ntheta; j++) {
		const double theta = M_PI * (j + 0.5) / ntheta;
		for(int i = 0; i < nphi; i++)
			grid[(size_t) j * nphi + i] = creal(orc_eval(a, l_max, polar, theta, 2.0 * M_PI * i / nphi));
	}
}

/* ------------------------------------------------------------------ */
/* peak finding (sh_series_extremize.c)                                */
/* ------------------------------------------------------------------ */

/* sh_series_extremize.c:168-241 */
double orc_find_near_minimum(const double complex *a, unsigned l_max, int polar, unsigned l_lowpass, double *theta, double *phi)
{
	unsigned L = l_max > l_lowpass ? l_lowpass : l_max;
	double complex *lo = malloc(orc_length(L, polar) * sizeof(*lo));
	orc_assign(lo, L, polar, a, l_max, polar);
	const int nt = 2 * (L + 1), np = nt;
	double complex *mesh = malloc((size_t) nt * np * sizeof(*mesh));
	orc_to_mesh(lo, L, polar, mesh);
	double *x = malloc(nt * sizeof(*x)), *w = malloc(nt * sizeof(*w));
	orc_gl_nodes(nt, x, w);
	double mn = INFINITY;
	*theta = *phi = NAN;
	for(int j = 0; j < nt; j++)
		for(int i = 0; i < np; i++) {
			const double v = creal(mesh[(size_t) j * np + i]);
			if(v < mn) {
				mn = v;
				*theta = acos(x[j]);
				*phi = 2. * M_PI * i / (double) np;
			}
		}
	free(w);
	free(x);
	free(mesh);
	free(lo);
	return mn;
}

/* sh_series_extremize.c:57-76 */
static void condition_theta_phi(double *theta, double *phi)
{
	*theta = fmod(*theta, 2 * M_PI);
	if(*theta < 0.)
		*theta += 2 * M_PI;
	if(*theta > M_PI) {
		*theta = 2. * M_PI - *theta;
		*phi += M_PI;
	}
	*phi = fmod(*phi, 2 * M_PI);
	if(*phi < 0.)
		*phi += 2 * M_PI;
}

/* Re f, d/dtheta Re f and (1/sin theta) d/dphi Re f at (theta, phi): the
 * value and the two gradient components the reference's dfunc() forms
 * (sh_series_extremize.c:115-150) from the series sin(theta) df/dtheta
 * and df/dphi (sh_series_deriv.c:531-543), here from the Legendre
 * derivative sin(theta) dP~_l^m/dtheta = l x P~_l^m
 * - sqrt((2l+1)(l^2-m^2)/(2l-1)) P~_{l-1}^m. */
static void re_value_grad(const double complex *a, unsigned l_max, int polar, double theta, double phi, double *f, double *u, double *v)
{
	const double x = cos(theta), st = sin(theta);
	double *P = malloc((l_max + 1) * sizeof(*P));
	double complex val = 0.0, dth = 0.0, dph = 0.0;
	const int mmax = polar ? 0 : (int) l_max;
	for(int m = -mmax; m <= mmax; m++) {
		const int am = abs(m);
		orc_sphPlm_array(l_max, am, x, P);
		const double sgn = (m < 0 && (am & 1)) ? -1.0 : 1.0;
		const double complex e = sgn * (cos(m * phi) + I * sin(m * phi));
		for(unsigned l = am; l <= l_max; l++) {
			const double complex c = a[orc_lmoffset(l_max, l, m)];
			const double p = P[l - am];
			const double pm1 = l > (unsigned) am ? P[l - 1 - am] : 0.0;
			const double s_dp = l * x * p - (l > (unsigned) am ? sqrt((2.0 * l + 1.0) * ((double) l * l - (double) m * m) / (2.0 * l - 1.0)) * pm1 : 0.0);
			val += c * e * p;
			dth += c * e * s_dp;
			dph += c * e * p * (I * m);
		}
	}
	free(P);
	*f = creal(val);
	*u = creal(dth) / st;
	*v = creal(dph) / st;
}

struct extremize_params {
	const double complex *a;
	unsigned l_max;
	int polar;
};

/* func() and dfunc() of sh_series_extremize.c:115-150: the series at the
 * conditioned co-ordinates, x = (theta, phi) left as the minimiser has it,
 * gradient (d/dtheta, (1/sin theta) d/dphi) -- the components along the
 * unit vectors, which are not the derivatives in the minimiser's
 * co-ordinates (theta, phi) */
static void extremize_fdf_ref(const double *xv, void *params, double *f, double *g)
{
	const struct extremize_params *ep = params;
	double t = xv[0], p = xv[1];
	condition_theta_phi(&t, &p);
	re_value_grad(ep->a, ep->l_max, ep->polar, t, p, f, &g[0], &g[1]);
}

/* the same value with the gradient in the co-ordinates themselves,
 * (d/dtheta, d/dphi) */
static void extremize_fdf_coord(const double *xv, void *params, double *f, double *g)
{
	const struct extremize_params *ep = params;
	double t = xv[0], p = xv[1];
	condition_theta_phi(&t, &p);
	re_value_grad(ep->a, ep->l_max, ep->polar, t, p, f, &g[0], &g[1]);
	g[1] *= sin(t);
}

/* the l <= 6 start, then the BFGS2 restatement of ref_shims/bfgs2.h (first
 * step pi/24, line tolerance 0.001, at most 100 iterations, stop at
 * |gradient| < 1e-3); minimises Re a; x left unconditioned */
static double minimise_bfgs2(const double complex *a, unsigned l_max, int polar, bfgs2_eval_fn fdf, double *theta, double *phi)
{
	double x0[2];
	if(isnan(orc_find_near_minimum(a, l_max, polar, 6, &x0[0], &x0[1])))
		return NAN;
	struct extremize_params ep = {a, l_max, polar};
	struct bfgs2 s;
	bfgs2_set(&s, 2, fdf, &ep, x0, M_PI / 24., 0.001);
	for(int iter = 0; iter < 100; iter++) {
		if(bfgs2_iterate(&s))
			break;
		if(sqrt(s.g[0] * s.g[0] + s.g[1] * s.g[1]) < 1e-3)
			break;
	}
	*theta = s.x[0];
	*phi = s.x[1];
	return s.f;
}

/* sh_series_real_minimum (sh_series_extremize.c:273-360) as the reference
 * runs it: its gradient convention, and (theta, phi) returned as the
 * minimiser leaves them (not conditioned). */
double orc_real_minimum_ref(const double complex *a, unsigned l_max, int polar, double *theta, double *phi)
{
	return minimise_bfgs2(a, l_max, polar, extremize_fdf_ref, theta, phi);
}

/* Maximum of Re a: the reference's method (l <= 6 start, BFGS2 with the
 * same parameters) on -a, with the gradient taken in the minimiser's own
 * co-ordinates so that the line search's slope is the true one; returns
 * max Re a and its conditioned co-ordinates. */
double orc_real_maximum(const double complex *a, unsigned l_max, int polar, double *theta, double *phi)
{
	const size_t len = orc_length(l_max, polar);
	double complex *neg = malloc(len * sizeof(*neg));
	for(size_t i = 0; i < len; i++)
		neg[i] = -a[i];
	double t, p;
	const double v = minimise_bfgs2(neg, l_max, polar, extremize_fdf_coord, &t, &p);
	free(neg);
	condition_theta_phi(&t, &p);
	*theta = t;
	*phi = p;
	return -v;
}
