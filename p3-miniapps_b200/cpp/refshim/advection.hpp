// Reference-facing C++ layer: namespace Advection
// (miniapps/vlp4d/thrust/advection.hpp:330-334), same signatures.
#ifndef VLP4D_B200_REFSHIM_ADVECTION_HPP
#define VLP4D_B200_REFSHIM_ADVECTION_HPP

#include "config.hpp"
#include "efield.hpp"
#include "types.hpp"

namespace Advection {
void advect_1D_x(Config *conf, const RealView4D &fn, RealView4D &fnp1, float64 dt);
void advect_1D_y(Config *conf, const RealView4D &fn, RealView4D &fnp1, float64 dt);
void advect_1D_vx(Config *conf, const RealView4D &fn, RealView4D &fnp1, Efield *ef, float64 dt);
void advect_1D_vy(Config *conf, const RealView4D &fn, RealView4D &fnp1, Efield *ef, float64 dt);
void print_fxvx(Config *conf, RealView4D &fn, int iter);
}  // namespace Advection

#endif
