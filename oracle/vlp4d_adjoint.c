/* Test infrastructure: FP64 discrete adjoint of the restated vlp4d step.
 *
 * The forward map is the restatement of vlp4d_oracle.c (orc_step, after
 * miniapps/vlp4d/openmp/timestep.hpp:11-55).  The adjoint here is written
 * independently of the CUDA library's formulation so that it can check it:
 *
 *  - every advection stage is transposed in scatter form: each output cell
 *    recomputes its own foot and weights exactly as the forward stage does
 *    (advect.hpp:112-317 restated) and pushes weight * lambda back onto its
 *    six taps;
 *  - the E-driven stages (vx, vy) add the derivative of their weights with
 *    respect to E: d = 2 + (hstar - (hmin + ipos*dh))/dh with
 *    hstar = hmin + fmod(hwidth + h - dt*E - hmin, hwidth), so
 *    dd/dE = -dt/dh inside a cell, and dw_k/dd is the derivative of the
 *    degree-5 polynomials of orc_lag_basis5 (product rule);
 *  - the field solve E = D(rho) is linear and translation-invariant (its
 *    Fourier filter does not depend on position; the rho -= 1 of cases
 *    10/20 only touches the mode the filter zeroes), so D is a circular
 *    convolution with the impulse response h = D(delta at the origin), and
 *    D^T g(q) = sum_p h(p - q) g(p), evaluated directly in real space.
 *
 * Objective: J(f) = dx*dy * sum_{ix,iy} (Ex^2 + Ey^2) with E = D(rho(f)),
 * the electric energy of the field solved from f.
 *
 * Sizes: the direct transposed field solve is O((nx*ny)^2) and the scatter
 * loops are serial, so this checker is meant for grids up to about 32^4.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "vlp4d_oracle.h"

static inline size_t aidx(const orc_domain *d, int ix, int iy, int ivx, int ivy) {
  return (size_t)ix + (size_t)d->n[0] * ((size_t)iy + (size_t)d->n[1] * ((size_t)ivx + (size_t)d->n[2] * (size_t)ivy));
}

/* d/dm of prod_i g_i(m), each g_i with derivative gp_i. */
static double prod_deriv(const double *g, const double *gp, int n) {
  double s = 0.;
  for (int i = 0; i < n; ++i) {
    double p = gp[i];
    for (int j = 0; j < n; ++j)
      if (j != i) p *= g[j];
    s += p;
  }
  return s;
}

/* Derivative of orc_lag_basis5 (advection.hpp:38-50) with respect to px.
 * With x = px - 2 the weights are
 *   w0 = -1/24 x (x-1) (x+1) (x-2) (x-1)
 *   w1 =  1/24 x (x-1) (x-2) (5x^2 + x - 8)
 *   w2 = -1/12 (x-1) (x-2) (x+1) (5x^2 - 3x - 6)
 *   w3 =  1/12 x (x+1) (x-2) (5x^2 - 7x - 4)
 *   w4 = -1/24 x (x-1) (x+1) (5x^2 - 11x - 2)
 *   w5 =  1/24 x (x-1) x (x+1) (x-2)                                  */
void orc_lag_basis5_deriv(double px, double dcoef[6]) {
  const double x = px - 2.;
  const double q1 = 5 * x * x + x - 8., q2 = 5 * x * x - 3 * x - 6., q3 = 5 * x * x - 7 * x - 4.,
               q4 = 5 * x * x - 11 * x - 2.;
  {
    const double g[5] = {x, x - 1., x + 1., x - 2., x - 1.}, gp[5] = {1, 1, 1, 1, 1};
    dcoef[0] = -1. / 24 * prod_deriv(g, gp, 5);
  }
  {
    const double g[4] = {x, x - 1., x - 2., q1}, gp[4] = {1, 1, 1, 10 * x + 1.};
    dcoef[1] = 1. / 24 * prod_deriv(g, gp, 4);
  }
  {
    const double g[4] = {x - 1., x - 2., x + 1., q2}, gp[4] = {1, 1, 1, 10 * x - 3.};
    dcoef[2] = -1. / 12 * prod_deriv(g, gp, 4);
  }
  {
    const double g[4] = {x, x + 1., x - 2., q3}, gp[4] = {1, 1, 1, 10 * x - 7.};
    dcoef[3] = 1. / 12 * prod_deriv(g, gp, 4);
  }
  {
    const double g[4] = {x, x - 1., x + 1., q4}, gp[4] = {1, 1, 1, 10 * x - 11.};
    dcoef[4] = -1. / 24 * prod_deriv(g, gp, 4);
  }
  {
    const double g[5] = {x, x - 1., x, x + 1., x - 2.}, gp[5] = {1, 1, 1, 1, 1};
    dcoef[5] = 1. / 24 * prod_deriv(g, gp, 5);
  }
}

/* The forward stages' per-cell foot (vlp4d_oracle.c, advect.hpp:139-304):
 * ipos (already minus LAG_OFFSET), the weights and the fractional position. */
static void afoot(double h, double disp, double hmin, double hwidth, double dh, double idh, int *ipos,
                  double coef[6], double *dpos) {
  const double hstar = hmin + fmod(hwidth + h - disp - hmin, hwidth);
  int ip = (int)floor((hstar - hmin) * idh);
  const double dd = 2 + idh * (hstar - (hmin + ip * dh));
  orc_lag_basis5(dd, coef);
  *ipos = ip - 2;
  *dpos = dd;
}

/* Transpose of orc_advect_x / orc_advect_y: lam_in = A^T lam_out. */
void orc_advect_x_T(const orc_domain *d, const double *lam_out, double *lam_in, double dt) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
  const double hmin = d->minp[0], hwidth = d->maxp[0] - d->minp[0];
  const double dh = d->dx[0], idh = 1. / d->dx[0];
  memset(lam_in, 0, sizeof(double) * (size_t)nx * ny * nvx * nvy);
  for (int ivy = 0; ivy < nvy; ++ivy)
    for (int ivx = 0; ivx < nvx; ++ivx)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          const double vx = d->minp[2] + ivx * d->dx[2];
          double coef[6], dd;
          int ipos;
          afoot(hmin + ix * dh, dt * vx, hmin, hwidth, dh, idh, &ipos, coef, &dd);
          const double l = lam_out[aidx(d, ix, iy, ivx, ivy)];
          for (int k = 0; k < 6; ++k) lam_in[aidx(d, (nx + ipos + k) % nx, iy, ivx, ivy)] += coef[k] * l;
        }
}

void orc_advect_y_T(const orc_domain *d, const double *lam_out, double *lam_in, double dt) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
  const double hmin = d->minp[1], hwidth = d->maxp[1] - d->minp[1];
  const double dh = d->dx[1], idh = 1. / d->dx[1];
  memset(lam_in, 0, sizeof(double) * (size_t)nx * ny * nvx * nvy);
  for (int ivy = 0; ivy < nvy; ++ivy)
    for (int ivx = 0; ivx < nvx; ++ivx)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          const double vy = d->minp[3] + ivy * d->dx[3];
          double coef[6], dd;
          int ipos;
          afoot(hmin + iy * dh, dt * vy, hmin, hwidth, dh, idh, &ipos, coef, &dd);
          const double l = lam_out[aidx(d, ix, iy, ivx, ivy)];
          for (int k = 0; k < 6; ++k) lam_in[aidx(d, ix, (ny + ipos + k) % ny, ivx, ivy)] += coef[k] * l;
        }
}

/* Transpose of orc_advect_vx (dim 2) / orc_advect_vy (dim 3) in f, plus the
 * gradient with respect to the driving field: g[ix + nx*iy] +=
 * sum over the column of lam_out * d(out)/dE, evaluated at the stage's input
 * f_in. */
static void advect_v_T(const orc_domain *d, int dim, const double *lam_out, const double *f_in,
                       const double *e, double dt, double *lam_in, double *g) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
  const int nv = d->n[dim];
  const double hmin = d->minp[dim], hwidth = d->maxp[dim] - d->minp[dim];
  const double dh = d->dx[dim], idh = 1. / d->dx[dim];
  memset(lam_in, 0, sizeof(double) * (size_t)nx * ny * nvx * nvy);
  memset(g, 0, sizeof(double) * (size_t)nx * ny);
  for (int ivy = 0; ivy < nvy; ++ivy)
    for (int ivx = 0; ivx < nvx; ++ivx)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          const int iv = dim == 2 ? ivx : ivy;
          const double ev = e[(size_t)ix + (size_t)nx * iy];
          double coef[6], dcoef[6], dd;
          int ipos;
          afoot(hmin + iv * dh, dt * ev, hmin, hwidth, dh, idh, &ipos, coef, &dd);
          orc_lag_basis5_deriv(dd, dcoef);
          const double l = lam_out[aidx(d, ix, iy, ivx, ivy)];
          double dsum = 0.;
          for (int k = 0; k < 6; ++k) {
            const int t = (nv + ipos + k) % nv;
            const size_t tap = dim == 2 ? aidx(d, ix, iy, t, ivy) : aidx(d, ix, iy, ivx, t);
            lam_in[tap] += coef[k] * l;
            dsum += dcoef[k] * f_in[tap];
          }
          g[(size_t)ix + (size_t)nx * iy] += l * dsum * (-dt * idh);
        }
}

void orc_advect_vx_T(const orc_domain *d, const double *lam_out, const double *f_in, const double *ex,
                     double dt, double *lam_in, double *gex) {
  advect_v_T(d, 2, lam_out, f_in, ex, dt, lam_in, gex);
}

void orc_advect_vy_T(const orc_domain *d, const double *lam_out, const double *f_in, const double *ey,
                     double dt, double *lam_in, double *gey) {
  advect_v_T(d, 3, lam_out, f_in, ey, dt, lam_in, gey);
}

/* lam_rho = D^T (gex, gey) for the field solve orc_field_poisson. */
void orc_field_poisson_T(const orc_domain *d, const double *gex, const double *gey, double *lam_rho) {
  const int nx = d->n[0], ny = d->n[1];
  const size_t n2 = (size_t)nx * ny;
  if (d->idcase == 2 || d->idcase == 6) {  /* analytic fields: E does not depend on rho */
    memset(lam_rho, 0, sizeof(double) * n2);
    return;
  }
  double *rho = (double *)calloc(n2, sizeof(double));
  double *hx = (double *)malloc(sizeof(double) * n2);
  double *hy = (double *)malloc(sizeof(double) * n2);
  rho[0] = 1.;
  orc_field_poisson(d, rho, hx, hy);
  for (int qy = 0; qy < ny; ++qy)
    for (int qx = 0; qx < nx; ++qx) {
      double s = 0.;
      for (int py = 0; py < ny; ++py)
        for (int px = 0; px < nx; ++px) {
          const size_t h = (size_t)((px - qx + nx) % nx) + (size_t)nx * (size_t)((py - qy + ny) % ny);
          const size_t p = (size_t)px + (size_t)nx * py;
          s += hx[h] * gex[p] + hy[h] * gey[p];
        }
      lam_rho[(size_t)qx + (size_t)nx * qy] = s;
    }
  free(hy);
  free(hx);
  free(rho);
}

/* J(f) and lam = dJ/df. */
void orc_energy_grad(const orc_domain *d, const double *f, double *J, double *lam) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
  const size_t n2 = (size_t)nx * ny;
  double *rho = (double *)malloc(sizeof(double) * n2 * 4);
  double *ex = rho + n2, *ey = ex + n2, *lr = ey + n2;
  orc_field_rho(d, f, rho);
  orc_field_poisson(d, rho, ex, ey);
  const double dxdy = d->dx[0] * d->dx[1];
  double e = 0.;
  for (size_t i = 0; i < n2; ++i) e += ex[i] * ex[i] + ey[i] * ey[i];
  *J = e * dxdy;
  for (size_t i = 0; i < n2; ++i) {
    ex[i] *= 2 * dxdy;
    ey[i] *= 2 * dxdy;
  }
  orc_field_poisson_T(d, ex, ey, lr);
  const double s = d->dx[2] * d->dx[3];
  for (int ivy = 0; ivy < nvy; ++ivy)
    for (int ivx = 0; ivx < nvx; ++ivx)
      for (size_t i = 0; i < n2; ++i) lam[i + n2 * ((size_t)ivx + (size_t)nvx * ivy)] = s * lr[i];
  free(rho);
}

/* lam_out = (step)^T lam_next at the state f_state (orc_step's sequence:
 * x, y (dt/2), rho, field, vx, vy (dt), x, y (dt/2)). */
void orc_step_adjoint(const orc_domain *d, const double *f_state, const double *lam_next, double *lam_out) {
  const int nx = d->n[0], ny = d->n[1], nvx = d->n[2], nvy = d->n[3];
  const size_t n2 = (size_t)nx * ny, n4 = n2 * nvx * nvy;
  const double dt = d->dt;
  double *a1 = (double *)malloc(sizeof(double) * n4 * 4);
  double *a2 = a1 + n4, *b1 = a2 + n4, *l = b1 + n4;
  double *rho = (double *)malloc(sizeof(double) * n2 * 6);
  double *ex = rho + n2, *ey = ex + n2, *gex = ey + n2, *gey = gex + n2, *lr = gey + n2;
  /* Forward recompute of the stage inputs. */
  orc_advect_x(d, f_state, a1, 0.5 * dt);
  orc_advect_y(d, a1, a2, 0.5 * dt);
  orc_field_rho(d, a2, rho);
  orc_field_poisson(d, rho, ex, ey);
  orc_advect_vx(d, a2, b1, ex, dt);
  /* Reverse sweep. */
  orc_advect_y_T(d, lam_next, l, 0.5 * dt);   /* lam c1 */
  orc_advect_x_T(d, l, lam_out, 0.5 * dt);    /* lam b2 */
  orc_advect_vy_T(d, lam_out, b1, ey, dt, l, gey);  /* lam b1 */
  orc_advect_vx_T(d, l, a2, ex, dt, lam_out, gex);  /* lam a2 (advection part) */
  orc_field_poisson_T(d, gex, gey, lr);
  const double s = d->dx[2] * d->dx[3];
  for (size_t v = 0; v < (size_t)nvx * nvy; ++v)
    for (size_t i = 0; i < n2; ++i) lam_out[i + n2 * v] += s * lr[i];
  orc_advect_y_T(d, lam_out, l, 0.5 * dt);    /* lam a1 */
  orc_advect_x_T(d, l, lam_out, 0.5 * dt);    /* lam f_state */
  free(rho);
  free(a1);
}

/* J(f_N) after nsteps steps from f0 (orc_step, diagnostics discarded) and
 * grad = dJ/df0.  Keeps every state (small grids only). */
void orc_adjoint_run(const orc_domain *d, const double *f0, int nsteps, double *J, double *grad) {
  const size_t n2 = (size_t)d->n[0] * d->n[1], n4 = n2 * d->n[2] * d->n[3];
  double *states = (double *)malloc(sizeof(double) * n4 * (size_t)(nsteps + 2));
  double *scratch = states + n4 * (size_t)(nsteps + 1);
  double *rho = (double *)malloc(sizeof(double) * n2 * 3);
  double *ex = rho + n2, *ey = ex + n2;
  memcpy(states, f0, sizeof(double) * n4);
  for (int s = 0; s < nsteps; ++s) {
    double nrj, mass;
    double *cur = states + n4 * (size_t)(s + 1);
    memcpy(cur, states + n4 * (size_t)s, sizeof(double) * n4);
    orc_step(d, cur, scratch, rho, ex, ey, &nrj, &mass);
  }
  double *lam = (double *)malloc(sizeof(double) * n4 * 2);
  double *lam2 = lam + n4;
  orc_energy_grad(d, states + n4 * (size_t)nsteps, J, lam);
  for (int s = nsteps - 1; s >= 0; --s) {
    orc_step_adjoint(d, states + n4 * (size_t)s, lam, lam2);
    memcpy(lam, lam2, sizeof(double) * n4);
  }
  memcpy(grad, lam, sizeof(double) * n4);
  free(lam);
  free(rho);
  free(states);
}
