/*
 * fftw3.h -- TEST INFRASTRUCTURE ONLY.  Project-written stand-in for the
 * subset of FFTW 3's public API that the reference's hot-path sources call
 * (correlator.c:216-244, sh_series_array.c:528-558, sh_series_trans.c:
 * 599-604, 686-692, 857-863), so that those sources compile unmodified
 * into the checker library under oracle/_ref.  Names and signatures are
 * FFTW's public interface; the transforms behind them are this project's
 * own (oracle/ref_shims/shim_fftw.c): unnormalised DFTs with FFTW's sign
 * convention, exp(sign * 2 pi i j k / n).  FFTW's planner semantics
 * (FFTW_MEASURE overwriting arrays while planning) are not reproduced:
 * planning never touches the arrays.
 */
#ifndef REF_SHIM_FFTW3_H
#define REF_SHIM_FFTW3_H

#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex fftw_complex;
typedef struct ref_shim_fftw_plan *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in, const int *inembed, int istride, int idist,
			     fftw_complex *out, const int *onembed, int ostride, int odist, int sign, unsigned flags);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in, const int *inembed, int istride, int idist,
				 fftw_complex *out, const int *onembed, int ostride, int odist, unsigned flags);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);

#ifdef __cplusplus
}
#endif

#endif
