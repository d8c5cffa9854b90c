// Per-line Lagrange-5 stencil of the semi-Lagrangian shift.
//
// The reference computes, for EVERY cell, the foot of the characteristic,
// its floor and the six weights (miniapps/vlp4d/thrust/advection.hpp:111-136
// and the three sibling functors).  Along one swept line the displacement is
// constant (dt*vx for x, dt*vy for y, dt*Ex(x,y) for vx, dt*Ey(x,y) for vy),
// so the foot's cell offset and its fractional position are the same for
// every cell of the line.  This header computes them ONCE per line, with the
// reference's formula evaluated at the line's first cell:
//
//   hstar = hmin + fmod(hwidth + h0 - disp - hmin, hwidth)      h0 = hmin
//   ip    = floor((hstar - hmin) / dh)
//   d     = 2 + (hstar - (hmin + ip*dh)) / dh                     in [2, 3)
//   w     = lag_basis(d)            (advection.hpp:38-50, LAG_ORDER 5)
//
// and cell i of the line reads taps (i + m + k) mod N, k = 0..5, m = ip - 2.
// Every floating-point operation is written with explicit round-to-nearest
// intrinsics on the device so no multiply-add is contracted: host and
// device produce the same bits, and both match the reference's CPU
// arithmetic for that cell.  The result differs from the reference's
// per-cell recomputation only by the rounding of the foot location
// (|d_i - d_0| ~ 1e-14), which the parity tests bound.
//
// The reference leaves displacements with disp > hwidth undefined (its
// fmod turns negative and the tap index goes below zero); here the foot is
// wrapped into [hmin, hmin + hwidth) so any displacement is periodic.
#pragma once

#include <cmath>

#ifdef __CUDA_ARCH__
#define VL_ADD(a, b) __dadd_rn((a), (b))
#define VL_SUB(a, b) __dsub_rn((a), (b))
#define VL_MUL(a, b) __dmul_rn((a), (b))
#else
#define VL_ADD(a, b) ((a) + (b))
#define VL_SUB(a, b) ((a) - (b))
#define VL_MUL(a, b) ((a) * (b))
#endif

namespace vlp4d {

// advection.hpp:38-50 (LAG_ORDER 5).  px is the fractional foot position
// measured from the first of the six nodes.
__host__ __device__ inline void lag_basis5(double px, double coef[6]) {
  const double loc0 = -1. / 24, loc1 = 1. / 24., loc2 = -1. / 12., loc3 = 1. / 12., loc4 = -1. / 24.,
               loc5 = 1. / 24.;
  const double pxm2 = VL_SUB(px, 2.);
  const double sqr = VL_MUL(pxm2, pxm2);
  const double p01 = VL_MUL(pxm2, VL_SUB(pxm2, 1.));
  const double p5s = VL_MUL(5., sqr);
  coef[0] = VL_MUL(VL_MUL(VL_MUL(VL_MUL(loc0, p01), VL_ADD(pxm2, 1.)), VL_SUB(pxm2, 2.)), VL_SUB(pxm2, 1.));
  coef[1] = VL_MUL(VL_MUL(VL_MUL(loc1, p01), VL_SUB(pxm2, 2.)), VL_SUB(VL_ADD(p5s, pxm2), 8.));
  coef[2] = VL_MUL(VL_MUL(VL_MUL(VL_MUL(loc2, VL_SUB(pxm2, 1.)), VL_SUB(pxm2, 2.)), VL_ADD(pxm2, 1.)),
                   VL_SUB(VL_SUB(p5s, VL_MUL(3., pxm2)), 6.));
  coef[3] = VL_MUL(VL_MUL(VL_MUL(VL_MUL(loc3, pxm2), VL_ADD(pxm2, 1.)), VL_SUB(pxm2, 2.)),
                   VL_SUB(VL_SUB(p5s, VL_MUL(7., pxm2)), 4.));
  coef[4] = VL_MUL(VL_MUL(VL_MUL(loc4, p01), VL_ADD(pxm2, 1.)), VL_SUB(VL_SUB(p5s, VL_MUL(11., pxm2)), 2.));
  coef[5] = VL_MUL(VL_MUL(VL_MUL(VL_MUL(loc5, p01), pxm2), VL_ADD(pxm2, 1.)), VL_SUB(pxm2, 2.));
}

// d/dpx of lag_basis5, for the reverse mode.  With x = px - 2 the weights
// are products of linear factors and one quadratic,
//   w0 = -1/24 x (x-1)^2 (x+1) (x-2)      w1 = 1/24 x (x-1) (x-2) (5x^2+x-8)
//   w2 = -1/12 (x-1) (x-2) (x+1) (5x^2-3x-6)
//   w3 =  1/12 x (x+1) (x-2) (5x^2-7x-4)  w4 = -1/24 x (x-1) (x+1) (5x^2-11x-2)
//   w5 =  1/24 x^2 (x-1) (x+1) (x-2),
// differentiated here with the product rule.
__host__ __device__ inline double prod_rule4(double a, double b, double c, double d, double da, double db, double dc,
                                             double dd) {
  return da * b * c * d + a * db * c * d + a * b * dc * d + a * b * c * dd;
}
__host__ __device__ inline void lag_basis5_deriv(double px, double dcoef[6]) {
  const double x = px - 2.;
  const double xm1 = x - 1., xp1 = x + 1., xm2 = x - 2.;
  // w0: x (x-1) (x+1) (x-2) * (x-1) ; w5: x (x-1) (x+1) (x-2) * x.
  const double p4 = x * xm1 * xp1 * xm2;
  const double dp4 = prod_rule4(x, xm1, xp1, xm2, 1., 1., 1., 1.);
  dcoef[0] = -1. / 24 * (dp4 * xm1 + p4);
  dcoef[1] = 1. / 24 * prod_rule4(x, xm1, xm2, 5 * x * x + x - 8., 1., 1., 1., 10 * x + 1.);
  dcoef[2] = -1. / 12 * prod_rule4(xm1, xm2, xp1, 5 * x * x - 3 * x - 6., 1., 1., 1., 10 * x - 3.);
  dcoef[3] = 1. / 12 * prod_rule4(x, xp1, xm2, 5 * x * x - 7 * x - 4., 1., 1., 1., 10 * x - 7.);
  dcoef[4] = -1. / 24 * prod_rule4(x, xm1, xp1, 5 * x * x - 11 * x - 2., 1., 1., 1., 10 * x - 11.);
  dcoef[5] = 1. / 24 * (dp4 * x + p4);
}

// FP32 difference weights of a line for the adjacent-difference form of
// stencil.cuh: v = (-w0, -(w0+w1), w3+w4+w5, w4+w5, w5), summed in FP64.
__host__ __device__ inline void weights_to_f32(const double w[6], float wf[6]) {
  wf[0] = (float)(-w[0]);
  wf[1] = (float)(-(w[0] + w[1]));
  wf[2] = (float)(w[3] + w[4] + w[5]);
  wf[3] = (float)(w[4] + w[5]);
  wf[4] = (float)w[5];
  wf[5] = 0.0f;
}

// The stencil of one swept line: cell i reads f[(i + m + k) mod n] * w[k].
struct LineStencil {
  int m;        // in [0, n)
  double w[6];
  double d;     // fractional foot position in [2, 3) the weights are evaluated at
};

// The transpose of a line's gather: cell j receives sum_k w[k] * l[(j - m - k) mod n],
// which is again a gather, with offset (-m - 5) mod n and the weights reversed.
__host__ __device__ inline LineStencil adjoint_stencil(const LineStencil &s, int n) {
  LineStencil a;
  a.m = (n - (s.m + 5) % n) % n;
  for (int k = 0; k < 6; ++k) a.w[k] = s.w[5 - k];
  a.d = s.d;
  return a;
}

// disp: physical displacement of the line (dt*v or dt*E); hmin/hmax: the
// swept dimension's minPhy/maxPhy; n: its number of points.
__host__ __device__ inline LineStencil line_stencil(double disp, double hmin, double hmax, int n) {
  const double hwidth = VL_SUB(hmax, hmin);
  const double dh = hwidth / (double)n;  // init.cpp:77-79 (a correctly rounded division on both sides)
  const double idh = 1. / dh;            // advection.hpp:97
  const double h0 = hmin;
  double hstar = VL_ADD(hmin, fmod(VL_SUB(VL_SUB(VL_ADD(hwidth, h0), disp), hmin), hwidth));
  if (hstar < hmin) hstar = VL_ADD(hstar, hwidth);  // disp > hwidth: outside the reference's range
  const int ip = (int)floor(VL_MUL(VL_SUB(hstar, hmin), idh));
  const double d = VL_ADD(2., VL_MUL(idh, VL_SUB(hstar, VL_ADD(hmin, VL_MUL((double)ip, dh)))));
  LineStencil s;
  lag_basis5(d, s.w);
  s.d = d;
  int m = (ip - 2) % n;
  if (m < 0) m += n;
  s.m = m;
  return s;
}

}  // namespace vlp4d
