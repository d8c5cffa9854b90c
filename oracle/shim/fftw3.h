/* Test infrastructure (oracle only): the subset of the FFTW3 C interface that
 * the reference's OpenMP FFT wrapper calls (lib/OpenMP_FFT.hpp:207-242 plans,
 * :271-420 executes, :599-652 1D wrappers).  FFTW itself is not installed
 * here; oracle/fftw_subset.c implements the double-precision entry points
 * from the definition of the discrete Fourier transform.  The single-
 * precision names are declared because the wrapper's float specialisation
 * names them, but the reference never instantiates it, so they have no
 * definitions.
 *
 * Semantics follow FFTW's documented conventions: transforms are
 * unnormalised, FFTW_FORWARD uses exp(-2*pi*i*j*k/n), FFTW_BACKWARD uses
 * exp(+2*pi*i*j*k/n), r2c writes n/2+1 outputs, c2r reads n/2+1 Hermitian
 * inputs and writes n reals.
 */
#ifndef ORACLE_SHIM_FFTW3_H
#define ORACLE_SHIM_FFTW3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef struct oracle_fft_plan_s *fftw_plan;
typedef struct oracle_fftf_plan_s *fftwf_plan;

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
void fftw_destroy_plan(fftw_plan p);
fftw_complex *fftw_alloc_complex(size_t n);
double *fftw_alloc_real(size_t n);
void fftw_free(void *p);

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned flags);
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out);
void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out);
void fftwf_destroy_plan(fftwf_plan p);
fftwf_complex *fftwf_alloc_complex(size_t n);
float *fftwf_alloc_real(size_t n);
void fftwf_free(void *p);

#ifdef __cplusplus
}
#endif

#endif
