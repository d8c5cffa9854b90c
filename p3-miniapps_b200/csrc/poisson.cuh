// The mode-wise spectral Poisson solve of the field solve (efield.cpp:68-99
// with the filter of efield.cpp:27-33), shared by the cuFFT path
// (k_poisson_solve) and the cluster solve (k_field_cluster): for the mode
// (ix1, ix2) of the half spectrum (kx = ix1 * kx0; ky = ix2 * ky0, negative
// branch for ix2 >= ny/2+1) and rho_hat r,
//   ex_hat = -i kx/k^2 r / (nx*ny), ey_hat = -i ky/k^2 r / (nx*ny),
//   phi_hat = r / k^2 / (nx*ny);  ky = 0 uses filter(kx) (0 at kx = 0).
#pragma once

#include <cufft.h>

namespace vlp4d {

__device__ __forceinline__ void poisson_mode(int ix1, int ix2, int nx2, double2 r, double kx0, double ky0,
                                             double normcoeff, double2 &e1, double2 &e2, double2 &r1) {
  const int nx2h = nx2 / 2 + 1;
  const double kx = ix1 * kx0;
  if (ix2 == 0) {
    const double filt = ix1 == 0 ? 0. : 1. / (kx * kx);
    e1.x = __dmul_rn(__dmul_rn(__dmul_rn(kx, r.y), filt), normcoeff);
    e1.y = __dmul_rn(__dmul_rn(__dmul_rn(-kx, r.x), filt), normcoeff);
    e2.x = 0.;
    e2.y = 0.;
    r1.x = __dmul_rn(__dmul_rn(r.x, filt), normcoeff);
    r1.y = __dmul_rn(__dmul_rn(r.y, filt), normcoeff);
  } else {
    const double ky = (ix2 < nx2h ? ix2 : ix2 - nx2) * ky0;
    const double k2 = __dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky));
    const double cx = -(kx / k2), cy = -(ky / k2);
    e1.x = __dmul_rn(-cx * r.y, normcoeff);
    e1.y = __dmul_rn(cx * r.x, normcoeff);
    e2.x = __dmul_rn(-cy * r.y, normcoeff);
    e2.y = __dmul_rn(cy * r.x, normcoeff);
    r1.x = __dmul_rn(r.x / k2, normcoeff);
    r1.y = __dmul_rn(r.y / k2, normcoeff);
  }
}

}  // namespace vlp4d
