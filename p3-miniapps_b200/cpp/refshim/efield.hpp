// Reference-facing C++ layer: Efield (miniapps/vlp4d/thrust/efield.hpp:10-37).
// Owns one vlp4d_ctx, which holds rho/phi, Ex, Ey, the FP64 FFT plans and
// the diagnostic history; rho_, ex_ and ey_ are views of its device fields.
// The context is registered for its Config so that the Advection functions,
// which the reference calls with the Config only, find it.
#ifndef VLP4D_B200_REFSHIM_EFIELD_HPP
#define VLP4D_B200_REFSHIM_EFIELD_HPP

#include "config.hpp"
#include "types.hpp"
#include "utils.hpp"

struct Efield {
  RealView2D rho_;
  RealView2D ex_;
  RealView2D ey_;
  RealView2D phi_;  // kept for interface parity; the reference never fills it either

  Efield(Config *conf, shape_nd<2> dim);
  virtual ~Efield();

  // efield.cpp:43-105: FFT solve of the current rho_ (xmax/ymax are the
  // domain maxima, as the reference passes them).
  void solve_poisson_fftw(float64 xmax, float64 ymax);

  vlp4d_ctx *ctx() const { return ctx_; }

 private:
  vlp4d_ctx *ctx_ = nullptr;
  const Config *conf_ = nullptr;
  DISALLOW_COPY_AND_ASSIGN(Efield);
};

namespace vlp4d_shim {
// The context registered for a Config by its Efield.
vlp4d_ctx *context_of(const Config *conf);
}  // namespace vlp4d_shim

#endif
