/*
 * shim_fftw.c -- TEST INFRASTRUCTURE ONLY.  This project's stand-in for the
 * FFTW 3 calls of the reference's hot-path sources (see fftw3.h), used only
 * to compile those sources unmodified into the checker library under
 * oracle/_ref.  Nothing in the product links it.
 *
 * Transforms are unnormalised DFTs, X[k] = sum_j x[j] exp(sign 2 pi i j k / n):
 *
 * - mixed-radix Cooley-Tukey (decimation in time, recursive, out of
 *   place) over the prime factors of n, each radix-r stage a direct r-point
 *   DFT; twiddles w^e = exp(sign 2 pi i e / n) are read from one table
 *   built in long double with the exact integer exponent, so every
 *   twiddle is correctly rounded;
 * - Bluestein's chirp-z method over a power-of-two transform when n has a
 *   prime factor above 127 (chirp phases from (j^2 mod 2n), exact);
 * - two exact identities checked first, in O(n): a constant sequence c
 *   transforms to (n c, 0, ..., 0) and a sequence that is zero except at
 *   j = 0 transforms to the constant x[0].  The reference's products of
 *   polar series go through full meshes whose rows are of exactly these
 *   two kinds (sh_series_product.c:269-329), so the identities keep the
 *   checker's l ~ 550 plan builds to minutes.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <fftw3.h>

typedef double complex cplx;

enum { KIND_C2C, KIND_R2C, KIND_C2R };

struct fft1d {
	int n;
	int sign;
	int nf;
	int f[64];
	cplx *tw;		/* tw[e] = exp(sign 2 pi i e / n), e < n */
	/* Bluestein */
	int M;
	cplx *chirp;		/* exp(sign pi i (j^2 mod 2n) / n), j < n */
	cplx *bhat;		/* forward M-point DFT of the conjugate chirp */
	struct fft1d *fwd, *bwd;
};

struct ref_shim_fftw_plan {
	int kind;
	int n, howmany;
	void *in, *out;
	int istride, idist, ostride, odist;
	struct fft1d *core;
	cplx *buf, *res;
};

static cplx expi_exact(long e, long n, int sign)
{
	/* exp(sign 2 pi i e / n) with e reduced into [0, n) */
	e %= n;
	if(e < 0)
		e += n;
	const long double ang = 2.0L * 3.14159265358979323846264338327950288L * (long double) e / (long double) n;
	const double c = (double) cosl(ang);
	const double s = (double) sinl(ang);
	return c + I * (sign < 0 ? -s : s);
}

static void fft1d_free(struct fft1d *p)
{
	if(!p)
		return;
	free(p->tw);
	free(p->chirp);
	free(p->bhat);
	fft1d_free(p->fwd);
	fft1d_free(p->bwd);
	free(p);
}

static void fft_rec(const struct fft1d *p, const cplx *x, long xs, cplx *X, int n, int fi, long twstep);

static struct fft1d *fft1d_new(int n, int sign)
{
	struct fft1d *p = calloc(1, sizeof(*p));
	if(!p)
		return NULL;
	p->n = n;
	p->sign = sign;
	int m = n, big = 0;
	for(int r = 2; m > 1; r++) {
		if((long) r * r > m)
			r = m;
		while(m % r == 0) {
			p->f[p->nf++] = r;
			if(r > 127)
				big = 1;
			m /= r;
		}
	}
	if(!big) {
		p->tw = malloc((size_t) n * sizeof(*p->tw));
		if(!p->tw) {
			fft1d_free(p);
			return NULL;
		}
		for(int e = 0; e < n; e++)
			p->tw[e] = expi_exact(e, n, sign);
		return p;
	}
	/* Bluestein */
	int M = 1;
	while(M < 2 * n - 1)
		M <<= 1;
	p->M = M;
	p->chirp = malloc((size_t) n * sizeof(*p->chirp));
	p->bhat = calloc((size_t) M, sizeof(*p->bhat));
	p->fwd = fft1d_new(M, -1);
	p->bwd = fft1d_new(M, +1);
	if(!p->chirp || !p->bhat || !p->fwd || !p->bwd) {
		fft1d_free(p);
		return NULL;
	}
	for(long j = 0; j < n; j++)
		p->chirp[j] = expi_exact((j * j) % (2L * n), 2L * n, sign);
	cplx *b = calloc((size_t) M, sizeof(*b));
	if(!b) {
		fft1d_free(p);
		return NULL;
	}
	b[0] = conj(p->chirp[0]);
	for(int j = 1; j < n; j++)
		b[j] = b[M - j] = conj(p->chirp[j]);
	fft_rec(p->fwd, b, 1, p->bhat, M, 0, 1);
	free(b);
	return p;
}

/* X[k] = sum_j x[j xs] W^(j k) for k < n, W = tw[twstep] (tw is the table of
 * the full length N = n * twstep); f[fi..] are the factors of n. */
static void fft_rec(const struct fft1d *p, const cplx *x, long xs, cplx *X, int n, int fi, long twstep)
{
	if(n == 1) {
		X[0] = x[0];
		return;
	}
	const int r = p->f[fi];
	const int m = n / r;
	for(int q = 0; q < r; q++)
		fft_rec(p, x + q * xs, xs * r, X + (long) q * m, m, fi + 1, twstep * r);
	const long N = (long) n * twstep;
	if(r == 2) {
		for(int k = 0; k < m; k++) {
			const cplx a = X[k];
			const cplx b = k ? X[m + k] * p->tw[k * twstep] : X[m];
			X[k] = a + b;
			X[m + k] = a - b;
		}
		return;
	}
	cplx t[128];
	const long rstep = N / r;
	for(int k = 0; k < m; k++) {
		for(int q = 0; q < r; q++)
			t[q] = (q && k) ? X[(long) q * m + k] * p->tw[(long) q * k * twstep] : X[(long) q * m + k];
		for(int s = 0; s < r; s++) {
			cplx acc = t[0];
			long idx = 0;
			const long step = (long) s * rstep;
			for(int q = 1; q < r; q++) {
				idx += step;
				if(idx >= N)
					idx -= N;
				acc += t[q] * p->tw[idx];
			}
			/* stored after all t[] are read: positions k + s m hold
			 * the inputs of this k only */
			X[k + (long) s * m] = acc;
		}
	}
}

/* out[k] = DFT of in[] (length p->n, contiguous); in and out distinct */
static void fft1d_exec(const struct fft1d *p, const cplx *in, cplx *out, cplx *scratch)
{
	const int n = p->n;
	int constant = 1, impulse = 1;
	for(int j = 1; j < n && (constant || impulse); j++) {
		if(in[j] != in[0])
			constant = 0;
		if(in[j] != 0)
			impulse = 0;
	}
	if(constant) {
		out[0] = n * in[0];
		for(int k = 1; k < n; k++)
			out[k] = 0;
		return;
	}
	if(impulse) {
		for(int k = 0; k < n; k++)
			out[k] = in[0];
		return;
	}
	if(!p->M) {
		fft_rec(p, in, 1, out, n, 0, 1);
		return;
	}
	const int M = p->M;
	cplx *a = scratch, *A = scratch + M;
	for(int j = 0; j < n; j++)
		a[j] = in[j] * p->chirp[j];
	for(int j = n; j < M; j++)
		a[j] = 0;
	fft_rec(p->fwd, a, 1, A, M, 0, 1);
	for(int j = 0; j < M; j++)
		A[j] *= p->bhat[j];
	fft_rec(p->bwd, A, 1, a, M, 0, 1);
	for(int k = 0; k < n; k++)
		out[k] = p->chirp[k] * a[k] / M;
}

static fftw_plan plan_new(int kind, int n, int howmany, void *in, int istride, int idist, void *out, int ostride, int odist, int sign)
{
	if(n <= 0 || howmany <= 0)
		return NULL;
	struct ref_shim_fftw_plan *p = calloc(1, sizeof(*p));
	if(!p)
		return NULL;
	p->kind = kind;
	p->n = n;
	p->howmany = howmany;
	p->in = in;
	p->out = out;
	p->istride = istride;
	p->idist = idist;
	p->ostride = ostride;
	p->odist = odist;
	p->core = fft1d_new(n, sign);
	const size_t scratch = (size_t) 2 * n + (p->core ? 2 * (size_t) p->core->M : 0);
	p->buf = malloc(scratch * sizeof(cplx));
	if(!p->core || !p->buf) {
		fftw_destroy_plan(p);
		return NULL;
	}
	p->res = p->buf + n;
	return p;
}

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in, const int *inembed, int istride, int idist,
			     fftw_complex *out, const int *onembed, int ostride, int odist, int sign, unsigned flags)
{
	(void) inembed;
	(void) onembed;
	(void) flags;
	if(rank != 1)
		return NULL;
	return plan_new(KIND_C2C, n[0], howmany, in, istride, idist, out, ostride, odist, sign);
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in, const int *inembed, int istride, int idist,
				 fftw_complex *out, const int *onembed, int ostride, int odist, unsigned flags)
{
	(void) inembed;
	(void) onembed;
	(void) flags;
	if(rank != 1)
		return NULL;
	return plan_new(KIND_R2C, n[0], howmany, in, istride, idist, out, ostride, odist, FFTW_FORWARD);
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{
	(void) flags;
	return plan_new(KIND_C2C, n, 1, in, 1, n, out, 1, n, sign);
}

fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags)
{
	(void) flags;
	return plan_new(KIND_R2C, n, 1, in, 1, n, out, 1, n / 2 + 1, FFTW_FORWARD);
}

fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags)
{
	(void) flags;
	return plan_new(KIND_C2R, n, 1, in, 1, n / 2 + 1, out, 1, n, FFTW_BACKWARD);
}

void fftw_execute(const fftw_plan p)
{
	const int n = p->n;
	cplx *scratch = p->core->M ? p->buf + 2 * n : NULL;
	for(int t = 0; t < p->howmany; t++) {
		switch(p->kind) {
		case KIND_C2C: {
			const cplx *in = (const cplx *) p->in + (long) t * p->idist;
			for(int j = 0; j < n; j++)
				p->buf[j] = in[(long) j * p->istride];
			fft1d_exec(p->core, p->buf, p->res, scratch);
			cplx *out = (cplx *) p->out + (long) t * p->odist;
			for(int k = 0; k < n; k++)
				out[(long) k * p->ostride] = p->res[k];
			break;
		}
		case KIND_R2C: {
			const double *in = (const double *) p->in + (long) t * p->idist;
			for(int j = 0; j < n; j++)
				p->buf[j] = in[(long) j * p->istride];
			fft1d_exec(p->core, p->buf, p->res, scratch);
			cplx *out = (cplx *) p->out + (long) t * p->odist;
			for(int k = 0; k <= n / 2; k++)
				out[(long) k * p->ostride] = p->res[k];
			break;
		}
		case KIND_C2R: {
			/* the input holds bins 0 .. n/2 of a Hermitian spectrum */
			const cplx *in = (const cplx *) p->in + (long) t * p->idist;
			for(int k = 0; k <= n / 2; k++)
				p->buf[k] = in[(long) k * p->istride];
			for(int k = n / 2 + 1; k < n; k++)
				p->buf[k] = conj(p->buf[n - k]);
			fft1d_exec(p->core, p->buf, p->res, scratch);
			double *out = (double *) p->out + (long) t * p->odist;
			for(int j = 0; j < n; j++)
				out[(long) j * p->ostride] = creal(p->res[j]);
			break;
		}
		}
	}
}

void fftw_destroy_plan(fftw_plan p)
{
	if(!p)
		return;
	fft1d_free(p->core);
	free(p->buf);
	free(p);
}
