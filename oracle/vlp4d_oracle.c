/* Test infrastructure: CPU oracle for the vlp4d step (see vlp4d_oracle.h).
 *
 * Plain-C restatement of yasahi-hpc/P3-miniapps miniapps/vlp4d/openmp.
 * Each function cites the reference lines it restates.  The per-cell
 * arithmetic keeps the reference's operation order (foot location, fmod
 * wrap, floor, offset, weights) so that the restatement agrees with the
 * compiled reference to the last bits on the same inputs; the only
 * reductions whose order differs are OpenMP sums, which the tests compare
 * with a tolerance.
 */
#include "vlp4d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846

static inline size_t idx4(const orc_domain *d, int ix, int iy, int ivx, int ivy) {
  return (size_t)ix + (size_t)d->n[0] * ((size_t)iy + (size_t)d->n[1] * ((size_t)ivx + (size_t)d->n[2] * (size_t)ivy));
}

/* miniapps/vlp4d/openmp/init.cpp:77-79: dx_ = (max - min) / N. */
void orc_domain_init(orc_domain *d, const int n[4], const double minp[4], const double maxp[4],
                     double dt, int idcase) {
  for (int i = 0; i < 4; ++i) {
    d->n[i] = n[i];
    d->minp[i] = minp[i];
    d->maxp[i] = maxp[i];
    d->dx[i] = (maxp[i] - minp[i]) / n[i];
  }
  d->dt = dt;
  d->idcase = idcase;
}

/* miniapps/vlp4d/openmp/advect.hpp:69-87 (LAG_ORDER 5: LAG_OFFSET 2,
 * LAG_PTS 6, odd order -> floor).  Degree-5 weights evaluated at px in [2,3). */
void orc_lag_basis5(double px, double coef[6]) {
  const double loc[6] = {-1. / 24, 1. / 24., -1. / 12., 1. / 12., -1. / 24., 1. / 24.};
  const double pxm2 = px - 2.;
  const double sqrpxm2 = pxm2 * pxm2;
  const double pxm2_01 = pxm2 * (pxm2 - 1.);
  coef[0] = loc[0] * pxm2_01 * (pxm2 + 1.) * (pxm2 - 2.) * (pxm2 - 1.);
  coef[1] = loc[1] * pxm2_01 * (pxm2 - 2.) * (5 * sqrpxm2 + pxm2 - 8.);
  coef[2] = loc[2] * (pxm2 - 1.) * (pxm2 - 2.) * (pxm2 + 1.) * (5 * sqrpxm2 - 3 * pxm2 - 6.);
  coef[3] = loc[3] * pxm2 * (pxm2 + 1.) * (pxm2 - 2.) * (5 * sqrpxm2 - 7 * pxm2 - 4.);
  coef[4] = loc[4] * pxm2_01 * (pxm2 + 1.) * (5 * sqrpxm2 - 11 * pxm2 - 2.);
  coef[5] = loc[5] * pxm2_01 * pxm2 * (pxm2 + 1.) * (pxm2 - 2.);
}

/* The foot of the characteristic and its stencil, as every advect_1D_*
 * computes it per cell (advect.hpp:139-150, 191-202, 242-253, 293-304):
 *   hstar = hmin + fmod(hwidth + h - disp - hmin, hwidth)
 *   ipos  = floor((hstar - hmin) / dh)
 *   d     = LAG_OFFSET + (hstar - (hmin + ipos*dh)) / dh
 * and the taps are (N + ipos - LAG_OFFSET + k) % N, k = 0..5. */
static inline void foot(double h, double disp, double hmin, double hwidth, double dh, double idh,
                        int *ipos_out, double coef[6]) {
  const double hstar = hmin + fmod(hwidth + h - disp - hmin, hwidth);
  int ipos1 = (int)floor((hstar - hmin) * idh);
  const double d_prev1 = 2 + idh * (hstar - (hmin + ipos1 * dh));
  ipos1 -= 2;
  orc_lag_basis5(d_prev1, coef);
  *ipos_out = ipos1;
}

/* advect.hpp:112-162: shift along x by dt*vx. */
void orc_advect_x(const orc_domain *d, const double *fn, double *fnp1, double dt) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
  const double hmin = d->minp[0], hwidth = d->maxp[0] - d->minp[0];
  const double dh = d->dx[0], idh = 1. / d->dx[0];
  const double minvx = d->minp[2], dvx = d->dx[2];
#pragma omp parallel for schedule(static) collapse(2)
  for (int ivy = 0; ivy < nvy; ++ivy)
    for (int ivx = 0; ivx < nvx; ++ivx)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          const double vx = minvx + ivx * dvx;
          const double x = hmin + ix * dh;
          double coef[6];
          int ipos;
          foot(x, dt * vx, hmin, hwidth, dh, idh, &ipos, coef);
          double acc = 0.;
          for (int k = 0; k < 6; ++k) acc += coef[k] * fn[idx4(d, (nx + ipos + k) % nx, iy, ivx, ivy)];
          fnp1[idx4(d, ix, iy, ivx, ivy)] = acc;
        }
}

/* advect.hpp:164-215: shift along y by dt*vy. */
void orc_advect_y(const orc_domain *d, const double *fn, double *fnp1, double dt) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
  const double hmin = d->minp[1], hwidth = d->maxp[1] - d->minp[1];
  const double dh = d->dx[1], idh = 1. / d->dx[1];
  const double minvy = d->minp[3], dvy = d->dx[3];
#pragma omp parallel for schedule(static) collapse(2)
  for (int ivy = 0; ivy < nvy; ++ivy)
    for (int ivx = 0; ivx < nvx; ++ivx)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          const double vy = minvy + ivy * dvy;
          const double y = hmin + iy * dh;
          double coef[6];
          int ipos;
          foot(y, dt * vy, hmin, hwidth, dh, idh, &ipos, coef);
          double acc = 0.;
          for (int k = 0; k < 6; ++k) acc += coef[k] * fn[idx4(d, ix, (ny + ipos + k) % ny, ivx, ivy)];
          fnp1[idx4(d, ix, iy, ivx, ivy)] = acc;
        }
}

/* advect.hpp:217-266: shift along vx by dt*Ex(x, y). */
void orc_advect_vx(const orc_domain *d, const double *fn, double *fnp1, const double *ex, double dt) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
  const double hmin = d->minp[2], hwidth = d->maxp[2] - d->minp[2];
  const double dh = d->dx[2], idh = 1. / d->dx[2];
#pragma omp parallel for schedule(static) collapse(2)
  for (int ivy = 0; ivy < nvy; ++ivy)
    for (int ivx = 0; ivx < nvx; ++ivx)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          const double vx = hmin + ivx * dh;
          double coef[6];
          int ipos;
          foot(vx, dt * ex[(size_t)ix + (size_t)nx * iy], hmin, hwidth, dh, idh, &ipos, coef);
          double acc = 0.;
          for (int k = 0; k < 6; ++k) acc += coef[k] * fn[idx4(d, ix, iy, (nvx + ipos + k) % nvx, ivy)];
          fnp1[idx4(d, ix, iy, ivx, ivy)] = acc;
        }
}

/* advect.hpp:269-317: shift along vy by dt*Ey(x, y). */
void orc_advect_vy(const orc_domain *d, const double *fn, double *fnp1, const double *ey, double dt) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
  const double hmin = d->minp[3], hwidth = d->maxp[3] - d->minp[3];
  const double dh = d->dx[3], idh = 1. / d->dx[3];
#pragma omp parallel for schedule(static) collapse(2)
  for (int ivy = 0; ivy < nvy; ++ivy)
    for (int ivx = 0; ivx < nvx; ++ivx)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          const double vy = hmin + ivy * dh;
          double coef[6];
          int ipos;
          foot(vy, dt * ey[(size_t)ix + (size_t)nx * iy], hmin, hwidth, dh, idh, &ipos, coef);
          double acc = 0.;
          for (int k = 0; k < 6; ++k) acc += coef[k] * fn[idx4(d, ix, iy, ivx, (nvy + ipos + k) % nvy)];
          fnp1[idx4(d, ix, iy, ivx, ivy)] = acc;
        }
}

/* miniapps/vlp4d/openmp/field.cpp:5-29: rho = dvx*dvy * sum over (ivy, ivx),
 * summed with ivy outer and ivx inner as the reference does. */
void orc_field_rho(const orc_domain *d, const double *fn, double *rho) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
  const double dvx = d->dx[2], dvy = d->dx[3];
#pragma omp parallel for schedule(static)
  for (int iy = 0; iy < ny; ++iy)
    for (int ix = 0; ix < nx; ++ix) {
      double sum = 0.;
      for (int ivy = 0; ivy < nvy; ++ivy)
        for (int ivx = 0; ivx < nvx; ++ivx) sum += fn[idx4(d, ix, iy, ivx, ivy)];
      rho[(size_t)ix + (size_t)nx * iy] = sum * dvx * dvy;
    }
}

/* ---- 2D real FFT (the reference uses FFTW through lib/OpenMP_FFT.hpp:
 * r2c along x for every y, then c2c along y for every kx; the inverse runs
 * c2c along y then c2r along x). */

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* In-place-safe complex DFT of length n with exponent sign*2*pi*i*j*k/n. */
static void cdft(int n, int sign, const double *xr, const double *xi, double *yr, double *yi) {
  const double two_pi = 2.0 * ORC_PI;
  double *ar = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  double *ai = ar + n;
  if (is_pow2(n)) {
    int bits = 0;
    while ((1 << bits) < n) ++bits;
    for (int j = 0; j < n; ++j) {
      int r = 0;
      for (int b = 0; b < bits; ++b) r |= ((j >> b) & 1) << (bits - 1 - b);
      ar[r] = xr[j];
      ai[r] = xi[j];
    }
    for (int len = 2; len <= n; len <<= 1) {
      const int half = len >> 1;
      for (int j = 0; j < half; ++j) {
        const double a = two_pi * (double)j / (double)len;
        const double wr = cos(a), wi = sign * sin(a);
        for (int i = 0; i < n; i += len) {
          const double br = ar[i + j + half], bi = ai[i + j + half];
          const double vr = br * wr - bi * wi, vi = br * wi + bi * wr;
          const double ur = ar[i + j], ui = ai[i + j];
          ar[i + j] = ur + vr;
          ai[i + j] = ui + vi;
          ar[i + j + half] = ur - vr;
          ai[i + j + half] = ui - vi;
        }
      }
    }
  } else {
    for (int k = 0; k < n; ++k) {
      double sr = 0., si = 0.;
      for (int j = 0; j < n; ++j) {
        const double a = two_pi * (double)(((long long)j * k) % n) / (double)n;
        const double wr = cos(a), wi = sign * sin(a);
        sr += xr[j] * wr - xi[j] * wi;
        si += xr[j] * wi + xi[j] * wr;
      }
      ar[k] = sr;
      ai[k] = si;
    }
  }
  memcpy(yr, ar, sizeof(double) * (size_t)n);
  memcpy(yi, ai, sizeof(double) * (size_t)n);
  free(ar);
}

void orc_rfft2(int nx1, int nx2, const double *in, double *hat) {
  const int nx1h = nx1 / 2 + 1;
  const int nmax = nx1 > nx2 ? nx1 : nx2;
  double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)nmax);
  double *xr = buf, *xi = buf + nmax, *yr = buf + 2 * nmax, *yi = buf + 3 * nmax;
  double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)nx1h * nx2);
  for (int j = 0; j < nx2; ++j) {
    for (int i = 0; i < nx1; ++i) { xr[i] = in[(size_t)i + (size_t)nx1 * j]; xi[i] = 0.; }
    cdft(nx1, -1, xr, xi, yr, yi);
    for (int i = 0; i < nx1h; ++i) {
      tmp[2 * ((size_t)i + (size_t)nx1h * j)] = yr[i];
      tmp[2 * ((size_t)i + (size_t)nx1h * j) + 1] = yi[i];
    }
  }
  for (int i = 0; i < nx1h; ++i) {
    for (int j = 0; j < nx2; ++j) {
      xr[j] = tmp[2 * ((size_t)i + (size_t)nx1h * j)];
      xi[j] = tmp[2 * ((size_t)i + (size_t)nx1h * j) + 1];
    }
    cdft(nx2, -1, xr, xi, yr, yi);
    for (int j = 0; j < nx2; ++j) {
      hat[2 * ((size_t)i + (size_t)nx1h * j)] = yr[j];
      hat[2 * ((size_t)i + (size_t)nx1h * j) + 1] = yi[j];
    }
  }
  free(tmp);
  free(buf);
}

void orc_irfft2(int nx1, int nx2, const double *hat, double *out) {
  const int nx1h = nx1 / 2 + 1;
  const int nmax = nx1 > nx2 ? nx1 : nx2;
  double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)nmax);
  double *xr = buf, *xi = buf + nmax, *yr = buf + 2 * nmax, *yi = buf + 3 * nmax;
  double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)nx1h * nx2);
  for (int i = 0; i < nx1h; ++i) {
    for (int j = 0; j < nx2; ++j) {
      xr[j] = hat[2 * ((size_t)i + (size_t)nx1h * j)];
      xi[j] = hat[2 * ((size_t)i + (size_t)nx1h * j) + 1];
    }
    cdft(nx2, +1, xr, xi, yr, yi);
    for (int j = 0; j < nx2; ++j) {
      tmp[2 * ((size_t)i + (size_t)nx1h * j)] = yr[j];
      tmp[2 * ((size_t)i + (size_t)nx1h * j) + 1] = yi[j];
    }
  }
  for (int j = 0; j < nx2; ++j) {
    /* Hermitian extension along x; imag parts of k=0 and k=n/2 do not
     * reach the real output (FFTW c2r convention). */
    for (int i = 0; i < nx1; ++i) {
      if (i < nx1h) {
        xr[i] = tmp[2 * ((size_t)i + (size_t)nx1h * j)];
        xi[i] = tmp[2 * ((size_t)i + (size_t)nx1h * j) + 1];
      } else {
        xr[i] = tmp[2 * ((size_t)(nx1 - i) + (size_t)nx1h * j)];
        xi[i] = -tmp[2 * ((size_t)(nx1 - i) + (size_t)nx1h * j) + 1];
      }
    }
    xi[0] = 0.;
    if (nx1 % 2 == 0) xi[nx1 / 2] = 0.;
    cdft(nx1, +1, xr, xi, yr, yi);
    for (int i = 0; i < nx1; ++i) out[(size_t)i + (size_t)nx1 * j] = yr[i];
  }
  free(tmp);
  free(buf);
}

/* miniapps/vlp4d/openmp/efield.cpp:50-104 (solve_poisson_fftw) together with
 * the filter built in the constructor (efield.cpp:28-37) and the case switch
 * of field_poisson (field.cpp:31-92).  kx0 = 2*pi/xmax uses maxPhy, not the
 * box length (field.cpp:94-97).  rho is overwritten with phi
 * (efield.cpp:101). */
void orc_field_poisson(const orc_domain *d, double *rho, double *ex, double *ey) {
  const int nx = d->n[0], ny = d->n[1];
  const double minx = d->minp[0], miny = d->minp[1], dx = d->dx[0], dy = d->dx[1];
  switch (d->idcase) {
    case 2:
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          ex[(size_t)ix + (size_t)nx * iy] = -(minx + ix * dx);
          ey[(size_t)ix + (size_t)nx * iy] = 0.;
        }
      return;
    case 6:
      /* field.cpp:55-68 writes ex from y in the OpenMP variant. */
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          ex[(size_t)ix + (size_t)nx * iy] = -(miny + iy * dy);
          ey[(size_t)ix + (size_t)nx * iy] = 0.;
        }
      return;
    case 10:
    case 20:
      for (size_t i = 0; i < (size_t)nx * ny; ++i) rho[i] -= 1.;
      break;
    default:
      break;
  }

  const int nx1h = nx / 2 + 1, nx2 = ny, nx2h = ny / 2 + 1;
  const double kx0 = 2 * ORC_PI / d->maxp[0];
  const double ky0 = 2 * ORC_PI / d->maxp[1];
  const double normcoeff = 1.0 / (double)(nx * ny);
  double *rho_hat = (double *)malloc(sizeof(double) * 2 * (size_t)nx1h * nx2);
  double *ex_hat = (double *)malloc(sizeof(double) * 2 * (size_t)nx1h * nx2);
  double *ey_hat = (double *)malloc(sizeof(double) * 2 * (size_t)nx1h * nx2);
  double *filter = (double *)malloc(sizeof(double) * (size_t)nx1h);
  filter[0] = 0.;
  for (int i = 1; i < nx1h; ++i) {
    const double kx = i * kx0;
    filter[i] = 1. / (kx * kx);
  }
  orc_rfft2(nx, ny, rho, rho_hat);
  for (int ix1 = 0; ix1 < nx1h; ++ix1) {
    const double kx = ix1 * kx0;
    for (int ix2 = 0; ix2 < nx2; ++ix2) {
      const size_t p = 2 * ((size_t)ix1 + (size_t)nx1h * ix2);
      const double rr = rho_hat[p], ri = rho_hat[p + 1];
      if (ix2 == 0) {
        /* -kx * I * rho_hat * filter * normcoeff */
        const double ar = kx * ri, ai = -kx * rr;
        ex_hat[p] = ar * filter[ix1] * normcoeff;
        ex_hat[p + 1] = ai * filter[ix1] * normcoeff;
        ey_hat[p] = 0.;
        ey_hat[p + 1] = 0.;
        rho_hat[p] = rr * filter[ix1] * normcoeff;
        rho_hat[p + 1] = ri * filter[ix1] * normcoeff;
      } else {
        const double ky = (ix2 < nx2h ? ix2 : ix2 - nx2) * ky0;
        const double k2 = kx * kx + ky * ky;
        /* -(k/k2) * I * rho_hat * normcoeff */
        const double cx = -(kx / k2), cy = -(ky / k2);
        ex_hat[p] = (-cx * ri) * normcoeff;
        ex_hat[p + 1] = (cx * rr) * normcoeff;
        ey_hat[p] = (-cy * ri) * normcoeff;
        ey_hat[p + 1] = (cy * rr) * normcoeff;
        rho_hat[p] = rr / k2 * normcoeff;
        rho_hat[p + 1] = ri / k2 * normcoeff;
      }
    }
  }
  orc_irfft2(nx, ny, rho_hat, rho);
  orc_irfft2(nx, ny, ex_hat, ex);
  orc_irfft2(nx, ny, ey_hat, ey);
  free(filter);
  free(ey_hat);
  free(ex_hat);
  free(rho_hat);
}

/* miniapps/vlp4d/openmp/diags.cpp:13-41: nrj = log(sqrt(sum |E|^2 dx dy))
 * (or -1e9 at or below 1e-30), mass = sum rho * dx * dy. */
void orc_diags(const orc_domain *d, const double *rho, const double *ex, const double *ey,
               double *nrj, double *mass) {
  const size_t n2 = (size_t)d->n[0] * d->n[1];
  double m = 0., e = 0.;
  for (size_t i = 0; i < n2; ++i) {
    m += rho[i];
    e += ex[i] * ex[i] + ey[i] * ey[i];
  }
  e = sqrt(e * d->dx[0] * d->dx[1]);
  *nrj = e > 1.e-30 ? log(e) : -1.e9;
  *mass = m * d->dx[0] * d->dx[1];
}

/* The vlp4d_mpi diagnostics, miniapps/vlp4d_mpi/thrust/Diags.cpp:17-66:
 * nrjx = sqrt(0.5 * sum Ex^2 * dx * dy), nrjy likewise with Ey. */
void orc_diags_mpi(const orc_domain *d, const double *ex, const double *ey, double *nrjx, double *nrjy) {
  const size_t n2 = (size_t)d->n[0] * d->n[1];
  double sx = 0., sy = 0.;
  for (size_t i = 0; i < n2; ++i) {
    sx += ex[i] * ex[i];
    sy += ey[i] * ey[i];
  }
  *nrjx = sqrt(0.5 * sx * d->dx[0] * d->dx[1]);
  *nrjy = sqrt(0.5 * sy * d->dx[0] * d->dx[1]);
}

/* Diags::computeL2norm, miniapps/vlp4d_mpi/thrust/Diags.cpp:68-92:
 * sqrt(sum f^2 * dx * dy * dvx * dvy) over the whole (single-rank) grid. */
double orc_l2norm(const orc_domain *d, const double *f) {
  const size_t n = (size_t)d->n[0] * d->n[1] * d->n[2] * d->n[3];
  double s = 0.;
  for (size_t i = 0; i < n; ++i) s += f[i] * f[i];
  return sqrt(s * d->dx[0] * d->dx[1] * d->dx[2] * d->dx[3]);
}

/* miniapps/vlp4d/openmp/timestep.hpp:11-55. */
void orc_step(const orc_domain *d, double *fn, double *fnp1, double *rho, double *ex, double *ey,
              double *nrj, double *mass) {
  orc_advect_x(d, fn, fnp1, 0.5 * d->dt);
  orc_advect_y(d, fnp1, fn, 0.5 * d->dt);
  orc_field_rho(d, fn, rho);
  orc_field_poisson(d, rho, ex, ey);
  orc_diags(d, rho, ex, ey, nrj, mass);
  orc_advect_vx(d, fn, fnp1, ex, d->dt);
  orc_advect_vy(d, fnp1, fn, ey, d->dt);
  orc_advect_x(d, fn, fnp1, 0.5 * d->dt);
  orc_advect_y(d, fnp1, fn, 0.5 * d->dt);
}

/* miniapps/vlp4d/openmp/vlp4d.cpp:58-74. */
void orc_run(const orc_domain *d, double *fn, double *fnp1, double *rho, double *ex, double *ey,
             int nsteps, double *nrj, double *mass) {
  orc_field_rho(d, fn, rho);
  orc_field_poisson(d, rho, ex, ey);
  orc_diags(d, rho, ex, ey, &nrj[0], &mass[0]);
  for (int it = 1; it <= nsteps; ++it) orc_step(d, fn, fnp1, rho, ex, ey, &nrj[it], &mass[it]);
}

/* Initial conditions.  SLD10: init.cpp:237-258; TSI20: init.cpp:261-288;
 * TSI20_MPI: miniapps/vlp4d_mpi/openmp/Init.cpp:249-277 (SLD10 there is
 * the same function as here);
 * CYL02/CYL05: init.cpp:146-234.  LANDAU_SUM and TWO_STREAM are the
 * perturbed Maxwellians of the benchmark configurations (amplitude amp,
 * wave number k, beam speed u). */
void orc_init_case(const orc_domain *d, double *f, int ic, double amp, double k, double u) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
#pragma omp parallel for schedule(static) collapse(2)
  for (int ivy = 0; ivy < nvy; ++ivy)
    for (int ivx = 0; ivx < nvx; ++ivx)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          const double x = d->minp[0] + ix * d->dx[0];
          const double y = d->minp[1] + iy * d->dx[1];
          const double vx = d->minp[2] + ivx * d->dx[2];
          const double vy = d->minp[3] + ivy * d->dx[3];
          double val = 0.;
          switch (ic) {
            case ORC_IC_SLD10: {
              const double sum = vx * vx + vy * vy;
              val = (1. / (2 * ORC_PI)) * exp(-0.5 * sum) * (1 + 0.05 * (cos(0.5 * x) * cos(0.5 * y)));
            } break;
            case ORC_IC_TSI20: {
              const double xi = 0.90, alpha = 0.05;
              const double sum = vx * vx + vy * vy;
              val = (1 + alpha * (cos(0.5 * x))) * 1 / (2 * ORC_PI) * ((2 - 2 * xi) / (3 - 2 * xi)) *
                    (1 + .5 * vx * vx / (1 - xi)) * exp(-.5 * sum);
            } break;
            case ORC_IC_TSI20_MPI: {
              const double vd = 2.4, vthx = 1.0, vthy = 0.5, ax = 0.05, ay = 0.25, kx = 0.2, ky = 0.2;
              val = 1. / (4 * ORC_PI * vthx * vthy) * (1 - ax * sin(kx * x) - ay * sin(ky * y)) *
                    (exp(-.5 * (pow((vx - vd) / vthx, 2) + pow(vy / vthy, 2))) +
                     exp(-.5 * (pow((vx + vd) / vthx, 2) + pow(vy / vthy, 2))));
            } break;
            case ORC_IC_CYL02:
            case ORC_IC_CYL05: {
              const double PERIOD = 0.5 * ORC_PI, AMPLI = 4;
              const double cc = 0.50 * (6. / 16.), rc = 0.50 * (4. / 16.);
              const double xx = ic == ORC_IC_CYL02 ? x : y;
              const double vv = ic == ORC_IC_CYL02 ? vx : vy;
              double hv = 0.0, hx = 0.0;
              if ((vv <= cc + rc) && (vv >= cc - rc)) hv = cos(PERIOD * ((vv - cc) / rc));
              else if ((vv <= -cc + rc) && (vv >= -cc - rc)) hv = -cos(PERIOD * ((vv + cc) / rc));
              if ((xx <= cc + rc) && (xx >= cc - rc)) hx = cos(PERIOD * ((xx - cc) / rc));
              else if ((xx <= -cc + rc) && (xx >= -cc - rc)) hx = -cos(PERIOD * ((xx + cc) / rc));
              val = AMPLI * hx * hv;
            } break;
            case ORC_IC_LANDAU_SUM: {
              const double m = exp(-0.5 * (vx * vx + vy * vy)) / (2 * ORC_PI);
              val = (1. + amp * cos(k * x) + amp * cos(k * y)) * m;
            } break;
            case ORC_IC_TWO_STREAM: {
              const double s = 1. / sqrt(2 * ORC_PI);
              const double mvy = s * exp(-0.5 * vy * vy);
              const double mb = 0.5 * (s * exp(-0.5 * (vx - u) * (vx - u)) + s * exp(-0.5 * (vx + u) * (vx + u)));
              val = (1. + amp * cos(k * x) + amp * cos(k * y)) * mb * mvy;
            } break;
            default:
              val = 0.;
          }
          f[idx4(d, ix, iy, ivx, ivy)] = val;
        }
}
