// Reference-facing C++ layer: miniapps/vlp4d/thrust/field.hpp:16-17.
#ifndef VLP4D_B200_REFSHIM_FIELD_HPP
#define VLP4D_B200_REFSHIM_FIELD_HPP

#include "config.hpp"
#include "diags.hpp"
#include "efield.hpp"
#include "types.hpp"

void field_rho(Config *conf, RealView4D &fn, Efield *ef);
void field_poisson(Config *conf, Efield *ef);

#endif
