// Reference-facing C++ layer: miniapps/vlp4d/thrust/init.hpp:8-9.
#ifndef VLP4D_B200_REFSHIM_INIT_HPP
#define VLP4D_B200_REFSHIM_INIT_HPP

#include "diags.hpp"
#include "efield.hpp"
#include "types.hpp"

void init(const char *file, Config *conf, RealView4D &fn, RealView4D &fnp1, Efield **ef, Diags **dg);
void finalize(Config *conf, Efield **ef, Diags **dg);

#endif
