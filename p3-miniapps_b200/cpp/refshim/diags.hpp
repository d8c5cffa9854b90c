// Reference-facing C++ layer: Diags (miniapps/vlp4d/thrust/diags.hpp:9-24).
// The history lives in the Efield's context on the device; save() writes
// the reference's nrj.out.
#ifndef VLP4D_B200_REFSHIM_DIAGS_HPP
#define VLP4D_B200_REFSHIM_DIAGS_HPP

#include "config.hpp"
#include "efield.hpp"
#include "types.hpp"
#include "utils.hpp"

struct Diags {
  explicit Diags(Config *conf);
  virtual ~Diags();

  void compute(Config *conf, Efield *ef, int iter);
  void save(Config *conf);

 private:
  DISALLOW_COPY_AND_ASSIGN(Diags);
};

#endif
