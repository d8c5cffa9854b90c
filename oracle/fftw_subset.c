/* Test infrastructure (oracle only).  A double-precision implementation of
 * the FFTW3 entry points declared in oracle/shim/fftw3.h, written from the
 * definition of the DFT:
 *
 *     X[k] = sum_{j=0}^{n-1} x[j] * exp(sign * 2*pi*i * j*k / n)
 *
 * Power-of-two lengths use an iterative radix-2 Cooley-Tukey transform
 * (decimation in time over a bit-reversed copy); other lengths use the
 * direct O(n^2) sum with a twiddle table indexed by (j*k) mod n.  Every
 * execute call works on private scratch, so concurrent calls on one plan
 * from several OpenMP threads are safe, which the reference relies on
 * (lib/OpenMP_FFT.hpp:271-420 call fftw_execute_* from inside
 * `#pragma omp parallel`).  The transforms are checked against numpy.fft
 * in tests/test_oracle_cpu.py.
 */
#include "shim/fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { KIND_C2C = 0, KIND_R2C = 1, KIND_C2R = 2 };

struct oracle_fft_plan_s {
  int n;
  int kind;
  int sign;
  int pow2;
  double *tw_re; /* exp(sign*2*pi*i*k/n), k = 0..n-1 */
  double *tw_im;
};

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static fftw_plan make_plan(int n, int kind, int sign) {
  if (n < 1) return NULL;
  fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
  p->n = n;
  p->kind = kind;
  p->sign = sign;
  p->pow2 = is_pow2(n);
  p->tw_re = (double *)malloc(sizeof(double) * (size_t)n);
  p->tw_im = (double *)malloc(sizeof(double) * (size_t)n);
  const double two_pi = 6.283185307179586476925286766559;
  for (int k = 0; k < n; ++k) {
    const double a = two_pi * (double)k / (double)n;
    p->tw_re[k] = cos(a);
    p->tw_im[k] = (double)sign * sin(a);
  }
  return p;
}

/* y = DFT_sign(x) for complex x given as separate re/im arrays. */
static void transform(const struct oracle_fft_plan_s *p, const double *xr, const double *xi,
                      double *yr, double *yi) {
  const int n = p->n;
  if (p->pow2) {
    int bits = 0;
    while ((1 << bits) < n) ++bits;
    for (int j = 0; j < n; ++j) {
      int r = 0;
      for (int b = 0; b < bits; ++b) r |= ((j >> b) & 1) << (bits - 1 - b);
      yr[r] = xr[j];
      yi[r] = xi[j];
    }
    for (int len = 2; len <= n; len <<= 1) {
      const int half = len >> 1;
      const int step = n / len;
      for (int i = 0; i < n; i += len) {
        for (int j = 0; j < half; ++j) {
          const double wr = p->tw_re[j * step], wi = p->tw_im[j * step];
          const double ur = yr[i + j], ui = yi[i + j];
          const double br = yr[i + j + half], bi = yi[i + j + half];
          const double vr = br * wr - bi * wi;
          const double vi = br * wi + bi * wr;
          yr[i + j] = ur + vr;
          yi[i + j] = ui + vi;
          yr[i + j + half] = ur - vr;
          yi[i + j + half] = ui - vi;
        }
      }
    }
  } else {
    for (int k = 0; k < n; ++k) {
      double sr = 0.0, si = 0.0;
      for (int j = 0; j < n; ++j) {
        const int t = (int)(((long long)j * (long long)k) % n);
        sr += xr[j] * p->tw_re[t] - xi[j] * p->tw_im[t];
        si += xr[j] * p->tw_im[t] + xi[j] * p->tw_re[t];
      }
      yr[k] = sr;
      yi[k] = si;
    }
  }
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
  (void)in; (void)out; (void)flags;
  return make_plan(n, KIND_C2C, sign < 0 ? -1 : +1);
}

fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags) {
  (void)in; (void)out; (void)flags;
  return make_plan(n, KIND_R2C, -1);
}

fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags) {
  (void)in; (void)out; (void)flags;
  return make_plan(n, KIND_C2R, +1);
}

void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out) {
  const int n = p->n;
  double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)n);
  double *xr = buf, *xi = buf + n, *yr = buf + 2 * n, *yi = buf + 3 * n;
  for (int j = 0; j < n; ++j) { xr[j] = in[j][0]; xi[j] = in[j][1]; }
  transform(p, xr, xi, yr, yi);
  for (int k = 0; k < n; ++k) { out[k][0] = yr[k]; out[k][1] = yi[k]; }
  free(buf);
}

void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out) {
  const int n = p->n;
  double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)n);
  double *xr = buf, *xi = buf + n, *yr = buf + 2 * n, *yi = buf + 3 * n;
  for (int j = 0; j < n; ++j) { xr[j] = in[j]; xi[j] = 0.0; }
  transform(p, xr, xi, yr, yi);
  for (int k = 0; k <= n / 2; ++k) { out[k][0] = yr[k]; out[k][1] = yi[k]; }
  free(buf);
}

/* Inverse of a Hermitian spectrum given by its first n/2+1 entries: the
 * missing entries are X[n-k] = conj(X[k]); the imaginary parts of X[0] and
 * (for even n) X[n/2] do not reach the real output. */
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) {
  const int n = p->n;
  double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)n);
  double *xr = buf, *xi = buf + n, *yr = buf + 2 * n, *yi = buf + 3 * n;
  const int nh = n / 2 + 1;
  for (int k = 0; k < nh; ++k) { xr[k] = in[k][0]; xi[k] = in[k][1]; }
  for (int k = nh; k < n; ++k) { xr[k] = in[n - k][0]; xi[k] = -in[n - k][1]; }
  xi[0] = 0.0;
  if (n % 2 == 0) xi[n / 2] = 0.0;
  transform(p, xr, xi, yr, yi);
  for (int j = 0; j < n; ++j) out[j] = yr[j];
  free(buf);
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  free(p->tw_re);
  free(p->tw_im);
  free(p);
}

fftw_complex *fftw_alloc_complex(size_t n) { return (fftw_complex *)malloc(sizeof(fftw_complex) * (n ? n : 1)); }
double *fftw_alloc_real(size_t n) { return (double *)malloc(sizeof(double) * (n ? n : 1)); }
void fftw_free(void *p) { free(p); }
