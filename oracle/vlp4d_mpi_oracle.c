/* Test infrastructure: CPU restatement of the reference's vlp4d_mpi step
 * (miniapps/vlp4d_mpi/openmp) for one process.  It is the checker for the
 * CUDA library's vlp4d_mpi entry points, never part of them: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  It is
 * pinned against the reference's own OpenMP vlp4d_mpi build
 * (oracle/ref_mpi_driver.cpp) and the committed fixtures in tests/golden/.
 *
 * Arrays are the reference's halo-extended views: extents n[d] + 6 with the
 * first index at -3 (HALO_PTS = 3, Config.hpp:7), FP64, layout_left, so
 * f(ix, iy, ivx, ivy) lives at (ix+3) + X*((iy+3) + Y*((ivx+3) + VX*(ivy+3)))
 * with X = nx + 6 and so on.  Every grid dimension must be at least 10
 * (MMAX + 2, Init.cpp:85-89): the boundary sums then read interior points
 * only.
 *
 * The scheme (Timestep.hpp:34-97, no LAG_ORDER: cubic B-splines):
 *   halo fill    periodic images, and in the outermost halo layer the sums
 *                sum_j alpha^j f(...) that stand in for the rest of the
 *                periodic line (Communication.hpp:756-896)
 *   spline xy    cubic B-spline prefilter along x then y (Spline.hpp:114-198)
 *   advect 2D    x, y shift by dt/2 through the 4x4 spline (Advection.hpp:
 *                87-164, 299-406); only its velocity moment is used
 *   field        rho, the one-process reduction, the Poisson solve
 *   spline vxvy  the prefilter along vx then vy (Spline.hpp:429-469)
 *   advect 4D    predictor-corrector foot with the field interpolated by
 *                3-point Lagrange, then the 4^4 spline interpolation
 *                (Advection.hpp:166-296, 409-498)
 *   field, diagnostics, L2 norm of the new state.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "vlp4d_oracle.h"

#define H 3      /* HALO_PTS */
#define MMAX 8   /* terms of a boundary sum (Config.hpp:8) */

static inline long hext(const orc_domain *d, int k) { return (long)d->n[k] + 2 * H; }

static inline size_t hidx(const orc_domain *d, int ix, int iy, int ivx, int ivy) {
  return (size_t)(ix + H) +
         (size_t)hext(d, 0) * ((size_t)(iy + H) + (size_t)hext(d, 1) * ((size_t)(ivx + H) + (size_t)hext(d, 2) * (size_t)(ivy + H)));
}

size_t orcm_size(const orc_domain *d) {
  return (size_t)hext(d, 0) * hext(d, 1) * hext(d, 2) * hext(d, 3);
}

/* Interior of a halo array to / from a plain n^4 array. */
void orcm_get_interior(const orc_domain *d, const double *fh, double *f) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
  for (int ivy = 0; ivy < nvy; ++ivy)
    for (int ivx = 0; ivx < nvx; ++ivx)
      for (int iy = 0; iy < ny; ++iy)
        memcpy(f + (size_t)nx * (iy + (size_t)ny * (ivx + (size_t)nvx * ivy)), fh + hidx(d, 0, iy, ivx, ivy),
               sizeof(double) * nx);
}

void orcm_set_interior(const orc_domain *d, double *fh, const double *f) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
  for (int ivy = 0; ivy < nvy; ++ivy)
    for (int ivx = 0; ivx < nvx; ++ivx)
      for (int iy = 0; iy < ny; ++iy)
        memcpy(fh + hidx(d, 0, iy, ivx, ivy), f + (size_t)nx * (iy + (size_t)ny * (ivx + (size_t)nvx * ivy)),
               sizeof(double) * nx);
}

static inline int wrap(int i, int n) { return ((i % n) + n) % n; }

/* Halo of one process (Communication.hpp:713-754 pack/unpack through the
 * local copy, with boundary_condition at :756-896 and the point lists of
 * listBoundary at :128-440).  A halo point whose coordinates all lie in
 * [-2, n+1] takes the periodic image.  A point in the outermost layer
 * (-3 or n+2) of the dimensions in B takes
 *     sum_{j_k = 1..MMAX, k in B} alpha^(sum j_k) f(r + sum_k s_k j_k e_k)
 * with s_k = -1 on the left layer and +1 on the right one, r_k = (c_k - s_k)
 * mod n_k for k in B and c_k mod n_k otherwise.  The sum runs with the
 * highest dimension of B in the outer loop and the powers of alpha built by
 * repeated products, as the reference does; points outer in several
 * dimensions keep the sum over all of them (the reference writes the lower
 * orders first and overwrites them). */
void orcm_halo_fill(const orc_domain *d, double *f) {
  const double alpha = sqrt(3.) - 2.;
  const int n[4] = {d->n[0], d->n[1], d->n[2], d->n[3]};
#pragma omp parallel for collapse(2) schedule(static)
  for (int cvy = -H; cvy < n[3] + H; ++cvy)
    for (int cvx = -H; cvx < n[2] + H; ++cvx)
      for (int cy = -H; cy < n[1] + H; ++cy)
        for (int cx = -H; cx < n[0] + H; ++cx) {
          const int c[4] = {cx, cy, cvx, cvy};
          int inside = 1;
          for (int k = 0; k < 4; ++k) inside &= (c[k] >= 0 && c[k] < n[k]);
          if (inside) continue;
          int B[4], s[4], m = 0, r[4];
          for (int k = 0; k < 4; ++k) {
            if (c[k] == -H || c[k] == n[k] + H - 1) {
              s[k] = c[k] == -H ? -1 : 1;
              B[m++] = k;
              r[k] = wrap(c[k] - s[k], n[k]);
            } else {
              s[k] = 0;
              r[k] = wrap(c[k], n[k]);
            }
          }
          double val;
          if (m == 0) {
            val = f[hidx(d, r[0], r[1], r[2], r[3])];
          } else {
            /* Odometer over j[0..m-1] (j[0]: lowest dimension, innermost),
             * weights w[l]: w[m-1] starts at alpha, an inner level starts
             * at alpha * (enclosing weight) and every level multiplies its
             * weight by alpha after each term. */
            int j[4] = {1, 1, 1, 1};
            double w[4];
            w[m - 1] = alpha;
            for (int l = m - 2; l >= 0; --l) w[l] = alpha * w[l + 1];
            double sum = 0.;
            for (;;) {
              int p[4] = {r[0], r[1], r[2], r[3]};
              for (int l = 0; l < m; ++l) p[B[l]] += s[B[l]] * j[l];
              sum += f[hidx(d, p[0], p[1], p[2], p[3])] * w[0];
              /* advance */
              int l = 0;
              w[0] *= alpha;
              while (l < m && ++j[l] > MMAX) {
                j[l] = 1;
                ++l;
                if (l < m) w[l] *= alpha;
              }
              if (l == m) break;
              for (int q = l - 1; q >= 0; --q) w[q] = alpha * w[q + 1];
            }
            val = sum;
          }
          f[hidx(d, cx, cy, cvx, cvy)] = val;
        }
}

/* The prefilter on one extended line (Spline.hpp:114-198, LONG_ENOUGH_BUFFER
 * form): e[0] and e[L+1] hold the boundary sums, e[1..L] the points
 * -2..n+1 (L = n + 4); e[1..L] are replaced by the spline coefficients,
 * e[0] and e[L+1] are left as they are.  tmp holds L values. */
static void spline_line(double *base, long stride, int n, double *tmp) {
  const double sqrt3 = sqrt(3.);
  const double alpha = sqrt3 - 2.;
  const double beta = sqrt3 * (1. - alpha * alpha);
  const int L = n + 4;
#define E(i) base[(long)(i) * stride]
  tmp[0] = E(0) + E(1);
  for (int k = 1; k < L; ++k) tmp[k] = E(1 + k) + alpha * tmp[k - 1];
  double acc = E(L + 1) + E(L);
  double ak = alpha;
  for (int k = 1; k < L; ++k) {
    acc += E(L - k) * ak;
    ak *= alpha;
  }
  E(L) = acc * sqrt3;
  for (int i = L - 1; i >= 1; --i) E(i) = beta * tmp[i - 1] + alpha * E(i + 1);
#undef E
}

/* Spline::computeCoeff_xy (Spline.hpp:384-426 -> :114-198): x lines for
 * every (y, vx, vy) of the extended array, then y lines for x in
 * [-2, nx+1]. */
void orcm_spline_xy(const orc_domain *d, double *f) {
  const long X = hext(d, 0), Y = hext(d, 1);
#pragma omp parallel for collapse(2) schedule(static)
  for (int ivy = -H; ivy < d->n[3] + H; ++ivy)
    for (int ivx = -H; ivx < d->n[2] + H; ++ivx) {
      double tmp[512];
      for (int iy = -H; iy < d->n[1] + H; ++iy) spline_line(f + hidx(d, -H, iy, ivx, ivy), 1, d->n[0], tmp);
      for (int ix = -H + 1; ix < d->n[0] + H - 1; ++ix) spline_line(f + hidx(d, ix, -H, ivx, ivy), X, d->n[1], tmp);
      (void)Y;
    }
}

/* Spline::computeCoeff_vxvy (Spline.hpp:429-469): through the transpose,
 * the same prefilter along vx (every vy) then along vy (vx in
 * [-2, nvx+1]), for every (x, y) of the extended array. */
void orcm_spline_vxvy(const orc_domain *d, double *f) {
  const long X = hext(d, 0), Y = hext(d, 1), VX = hext(d, 2);
#pragma omp parallel for collapse(2) schedule(static)
  for (int iy = -H; iy < d->n[1] + H; ++iy)
    for (int ix = -H; ix < d->n[0] + H; ++ix) {
      double tmp[512];
      for (int ivy = -H; ivy < d->n[3] + H; ++ivy) spline_line(f + hidx(d, ix, iy, -H, ivy), X * Y, d->n[2], tmp);
      for (int ivx = -H + 1; ivx < d->n[2] + H - 1; ++ivx)
        spline_line(f + hidx(d, ix, iy, ivx, -H), X * Y * VX, d->n[3], tmp);
    }
}

/* Cubic B-spline weights at fractional offset w (Advection.hpp:127-144). */
static inline void bspline_weights(double w, double eta[4]) {
  const double e3 = (1. / 6.) * w * w * w;
  const double e0 = (1. / 6.) + 0.5 * w * (w - 1.) - e3;
  const double e2 = w + e0 - 2. * e3;
  const double e1 = 1. - e0 - e2 - e3;
  eta[0] = e0;
  eta[1] = e1;
  eta[2] = e2;
  eta[3] = e3;
}

/* Advection::advect_2D_xy (Advection.hpp:299-406 with interp_2D at :87-164,
 * spline branch): tmp receives a copy of f (spline coefficients), f's
 * interior the interpolated values at the feet (x - dt vx, y - dt vy).
 * Returns the number of feet outside the interpolation range (the
 * reference then stops: "Time step is too large"). */
int orcm_advect_2d(const orc_domain *d, double *f, double *tmp, double dt) {
  memcpy(tmp, f, sizeof(double) * orcm_size(d));
  const double inv_dx0 = 1. / d->dx[0], inv_dx1 = 1. / d->dx[1];
  int err = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : err)
  for (int ivy = 0; ivy < d->n[3]; ++ivy)
    for (int ivx = 0; ivx < d->n[2]; ++ivx)
      for (int iy = 0; iy < d->n[1]; ++iy)
        for (int ix = 0; ix < d->n[0]; ++ix) {
          const double x = d->minp[0] + ix * d->dx[0];
          const double y = d->minp[1] + iy * d->dx[1];
          const double vx = d->minp[2] + ivx * d->dx[2];
          const double vy = d->minp[3] + ivy * d->dx[3];
          const double xs = x - dt * vx, ys = y - dt * vy;
          const double fx = (xs - d->minp[0]) * inv_dx0;
          const double fy = (ys - d->minp[1]) * inv_dx1;
          const int i0 = (int)floor(fx), i1 = (int)floor(fy);
          double ex[4], ey[4];
          bspline_weights(fx - (double)i0, ex);
          bspline_weights(fy - (double)i1, ey);
          double val = 0.;
          if (i0 < -1 || i0 > d->n[0] - 1 || i1 < -1 || i1 > d->n[1] - 1) {
            ++err;
          } else {
            for (int ky = 0; ky < 4; ++ky) {
              double s = 0.;
              for (int kx = 0; kx < 4; ++kx) s += ex[kx] * tmp[hidx(d, i0 - 1 + kx, i1 - 1 + ky, ivx, ivy)];
              val += ey[ky] * s;
            }
          }
          f[hidx(d, ix, iy, ivx, ivy)] = val;
        }
  return err;
}

/* 3-point Lagrange weights (Advection.hpp:26-30). */
static inline void lag3(double p, double c[3]) {
  c[0] = .5 * (p - 1.) * (p - 2.);
  c[1] = -1. * (p) * (p - 2.);
  c[2] = .5 * (p) * (p - 1.);
}

/* The 4D foot of cell (ix, iy, ivx, ivy) (computeFeet, Advection.hpp:166-218):
 * a half-step predictor at the cell's own field, the field interpolated
 * (periodic 3x3 Lagrange) at the predicted (x, y), then the full step. */
static void foot4d(const orc_domain *d, const double *ex, const double *ey, int ix, int iy, int ivx, int ivy,
                   double xs[4]) {
  const int nx = d->n[0], ny = d->n[1];
  const double x = d->minp[0] + ix * d->dx[0];
  const double y = d->minp[1] + iy * d->dx[1];
  const double vx = d->minp[2] + ivx * d->dx[2];
  const double vy = d->minp[3] + ivy * d->dx[3];
  const double dt = d->dt;
  double t[4];
  t[0] = x - 0.5 * dt * vx;
  t[1] = y - 0.5 * dt * vy;
  t[2] = vx - 0.5 * dt * ex[ix + (size_t)nx * iy];
  t[3] = vy - 0.5 * dt * ey[ix + (size_t)nx * iy];
  int ip[2];
  double c[2][3];
  for (int j = 0; j < 2; ++j) {
    t[j] = (1. / d->dx[j]) * (t[j] - d->minp[j]);
    ip[j] = (int)(round(t[j]) - 1);
    lag3(t[j] - ip[j], c[j]);
  }
  double e1 = 0., e2 = 0.;
  for (int k1 = 0; k1 <= 2; ++k1)
    for (int k0 = 0; k0 <= 2; ++k0) {
      const int jx = (nx + ip[0] + k0) % nx, jy = (ny + ip[1] + k1) % ny;
      e1 += c[0][k0] * c[1][k1] * ex[jx + (size_t)nx * jy];
      e2 += c[0][k0] * c[1][k1] * ey[jx + (size_t)nx * jy];
    }
  t[2] = vx - 0.5 * dt * e1;
  t[3] = vy - 0.5 * dt * e2;
  xs[0] = x - dt * t[2];
  xs[1] = y - dt * t[3];
  const double w2 = d->maxp[2] - d->minp[2], w3 = d->maxp[3] - d->minp[3];
  xs[2] = fmax(fmin(vx - dt * e1, d->minp[2] + w2), d->minp[2]);
  xs[3] = fmax(fmin(vy - dt * e2, d->minp[3] + w3), d->minp[3]);
}

/* Advection::advect_4D (Advection.hpp:409-498, interp_4D at :221-296 spline
 * branch) with dt = d->dt: tmp receives a copy of fn (4D spline
 * coefficients), fn's interior the interpolated values.  Returns the number
 * of feet outside [min - h, min + (n-1) h + h] in some dimension. */
int orcm_advect_4d(const orc_domain *d, const double *ex, const double *ey, double *fn, double *tmp) {
  memcpy(tmp, fn, sizeof(double) * orcm_size(d));
  int err = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : err)
  for (int ivy = 0; ivy < d->n[3]; ++ivy)
    for (int ivx = 0; ivx < d->n[2]; ++ivx)
      for (int iy = 0; iy < d->n[1]; ++iy)
        for (int ix = 0; ix < d->n[0]; ++ix) {
          double xs[4];
          foot4d(d, ex, ey, ix, iy, ivx, ivy, xs);
          int bad = 0;
          for (int j = 0; j < 4; ++j) {
            const double lo = d->minp[j] - d->dx[j];
            const double hi = d->minp[j] + (d->n[j] - 1) * d->dx[j] + d->dx[j];
            bad += (xs[j] < lo || xs[j] > hi);
          }
          if (bad) {
            /* The reference stops the run; the checker only counts. */
            err += bad;
            fn[hidx(d, ix, iy, ivx, ivy)] = 0.;
            continue;
          }
          int ip[4];
          double eta[4][4];
          for (int j = 0; j < 4; ++j) {
            const double g = (1. / d->dx[j]) * (xs[j] - d->minp[j]);
            ip[j] = (int)floor(g);
            bspline_weights(g - ip[j], eta[j]);
          }
          double v = 0.;
          for (int k3 = 0; k3 < 4; ++k3)
            for (int k2 = 0; k2 < 4; ++k2) {
              double s2 = 0.;
              for (int k1 = 0; k1 < 4; ++k1) {
                double s3 = 0.;
                const double *row = tmp + hidx(d, ip[0] - 1, ip[1] + k1 - 1, ip[2] + k2 - 1, ip[3] + k3 - 1);
                for (int k0 = 0; k0 < 4; ++k0) s3 += eta[0][k0] * row[k0];
                s2 += s3 * eta[1][k1];
              }
              v += s2 * eta[2][k2] * eta[3][k3];
            }
          fn[hidx(d, ix, iy, ivx, ivy)] = v;
        }
  return err;
}

/* field_rho (Field.cpp:5-55) on the interior of a halo array. */
void orcm_field_rho(const orc_domain *d, const double *f, double *rho) {
  const int nx = d->n[0], ny = d->n[1];
#pragma omp parallel for schedule(static)
  for (int iy = 0; iy < ny; ++iy)
    for (int ix = 0; ix < nx; ++ix) {
      double s = 0.;
      for (int ivy = 0; ivy < d->n[3]; ++ivy)
        for (int ivx = 0; ivx < d->n[2]; ++ivx) s += f[hidx(d, ix, iy, ivx, ivy)];
      rho[ix + (size_t)nx * iy] = s * d->dx[2] * d->dx[3];
    }
}

/* Diags::computeL2norm (Diags.cpp:50-76) over the interior. */
double orcm_l2norm(const orc_domain *d, const double *f) {
  double s = 0.;
  for (int ivy = 0; ivy < d->n[3]; ++ivy)
    for (int ivx = 0; ivx < d->n[2]; ++ivx)
      for (int iy = 0; iy < d->n[1]; ++iy)
        for (int ix = 0; ix < d->n[0]; ++ix) {
          const double v = f[hidx(d, ix, iy, ivx, ivy)];
          s += v * v;
        }
  return sqrt(s * d->dx[0] * d->dx[1] * d->dx[2] * d->dx[3]);
}

/* Diags::compute (Diags.cpp:16-48): diag[0..3] = nrj, nrjx, nrjy, mass. */
static void diags_all(const orc_domain *d, const double *rho, const double *ex, const double *ey, double diag[4]) {
  orc_diags(d, rho, ex, ey, &diag[0], &diag[3]);
  orc_diags_mpi(d, ex, ey, &diag[1], &diag[2]);
}

/* field_rho + field_reduce + field_poisson (Field.cpp): rho is overwritten
 * with phi, as in the reference. */
static void field_all(const orc_domain *d, const double *f, double *rho, double *ex, double *ey) {
  orcm_field_rho(d, f, rho);
  orc_field_poisson(d, rho, ex, ey);
}

/* The initial field, diagnostics and L2 norm before the time loop
 * (Vlp4d.cpp:31-35).  out[0..4] = nrj, nrjx, nrjy, mass, l2norm. */
void orcm_start(const orc_domain *d, const double *fn, double *rho, double *ex, double *ey, double out[5]) {
  field_all(d, fn, rho, ex, ey);
  diags_all(d, rho, ex, ey, out);
  out[4] = orcm_l2norm(d, fn);
}

/* onetimestep (Timestep.hpp:34-97) and the swap of Vlp4d.cpp:46: fn holds
 * the state before and after; fnp1 and tmp are scratch halo arrays.
 * half[0..3] receives the diagnostics of the mid-step field, out[0..4]
 * those of the end-of-step field and the L2 norm.  Returns the number of
 * out-of-range feet of the two advections. */
int orcm_step(const orc_domain *d, double *fn, double *fnp1, double *tmp, double *rho, double *ex, double *ey,
              double half[4], double out[5]) {
  orcm_halo_fill(d, fn);
  orcm_spline_xy(d, fn);
  memcpy(fnp1, fn, sizeof(double) * orcm_size(d));
  int err = orcm_advect_2d(d, fn, tmp, 0.5 * d->dt);
  field_all(d, fn, rho, ex, ey);
  diags_all(d, rho, ex, ey, half);
  orcm_spline_vxvy(d, fnp1);
  err += orcm_advect_4d(d, ex, ey, fnp1, fn);
  field_all(d, fnp1, rho, ex, ey);
  diags_all(d, rho, ex, ey, out);
  out[4] = orcm_l2norm(d, fnp1);
  /* swap: the new state goes back into fn (the reference swaps views). */
  memcpy(fn, fnp1, sizeof(double) * orcm_size(d));
  return err;
}

/* Initial condition on the interior (Init.cpp:126-277); the halo is zero,
 * as after init() (Init.cpp:370-372). */
void orcm_init_case(const orc_domain *d, double *fh, int ic) {
  const size_t n = (size_t)d->n[0] * d->n[1] * d->n[2] * d->n[3];
  double *f = (double *)malloc(sizeof(double) * n);
  orc_init_case(d, f, ic, 0., 0., 0.);
  memset(fh, 0, sizeof(double) * orcm_size(d));
  orcm_set_interior(d, fh, f);
  free(f);
}
