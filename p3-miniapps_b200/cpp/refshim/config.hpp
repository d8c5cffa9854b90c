// Reference-facing C++ layer: the reference's Config/Domain/Physics
// (miniapps/vlp4d/thrust/config.hpp:8-36), same fields and meanings.
#ifndef VLP4D_B200_REFSHIM_CONFIG_HPP
#define VLP4D_B200_REFSHIM_CONFIG_HPP

#include "types.hpp"

static constexpr size_t DIMENSION = 4;

struct Domain {
  shape_nd<DIMENSION> nxmax_;  // points per dimension: x, y, vx, vy
  int nbiter_, ifreq_;         // number of steps, diagnostic frequency
  int idcase_;                 // test case (selects initial condition and field_poisson branch)
  float64 minPhy_[DIMENSION];
  float64 maxPhy_[DIMENSION];
  float64 dt_;
  float64 dx_[DIMENSION];
  char limitCondition_[DIMENSION];
  int fxvx_;
};

struct Physics {
  float64 z_, S_, omega02_, vbeam_, beta_, psi_, eps0_, echarge_, mass_;
};

struct Config {
  Physics phys_;
  Domain dom_;
};

namespace vlp4d_shim {
// The C ABI's domain description of a Config.
inline vlp4d_domain to_domain(const Config *conf) {
  vlp4d_domain d{};
  for (size_t i = 0; i < DIMENSION; ++i) {
    d.nxmax[i] = conf->dom_.nxmax_[i];
    d.min_phy[i] = conf->dom_.minPhy_[i];
    d.max_phy[i] = conf->dom_.maxPhy_[i];
  }
  d.dt = conf->dom_.dt_;
  d.nbiter = conf->dom_.nbiter_;
  d.ifreq = conf->dom_.ifreq_;
  d.idcase = conf->dom_.idcase_;
  d.fxvx = conf->dom_.fxvx_;
  return d;
}
}  // namespace vlp4d_shim

#endif
