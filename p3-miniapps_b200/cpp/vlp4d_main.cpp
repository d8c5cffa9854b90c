// vlp4d_b200 driver: the flow of the reference's main()
// (miniapps/vlp4d/thrust/vlp4d.cpp:33-81) on the reference-facing C++ layer.
//
//   vlp4d_b200 <deck> [--fused]
//
// Without --fused every step runs the reference's stage sequence
// (timestep.hpp:14-67) through the 1D entry points, timed per stage with the
// reference's labels; with --fused each step is one vlp4d_step (three fused
// passes).  Writes nrj.out and prints "label seconds [s], calls calls".
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "refshim/advection.hpp"
#include "refshim/config.hpp"
#include "refshim/diags.hpp"
#include "refshim/efield.hpp"
#include "refshim/field.hpp"
#include "refshim/init.hpp"

namespace {

struct StageTimer {
  std::string label;
  double seconds = 0;
  int calls = 0;
  std::chrono::steady_clock::time_point t0;
  void begin() { t0 = std::chrono::steady_clock::now(); }
  void end() {
    synchronize();
    seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    ++calls;
  }
};

enum { kTotal, kMainLoop, kX, kY, kVx, kVy, kField, kFourier, kDiag, kStep, kCount };
const char *kLabels[kCount] = {"total", "MainLoop", "advec1D_x", "advec1D_y", "advec1D_vx",
                               "advec1D_vy", "field", "Fourier", "diag", "fused_step"};

void staged_step(Config *conf, RealView4D &fn, RealView4D &fnp1, Efield *ef, Diags *dg, StageTimer *t, int iter) {
  const float64 dt = conf->dom_.dt_;
  t[kX].begin(); Advection::advect_1D_x(conf, fn, fnp1, 0.5 * dt); t[kX].end();
  t[kY].begin(); Advection::advect_1D_y(conf, fnp1, fn, 0.5 * dt); t[kY].end();
  t[kField].begin(); field_rho(conf, fn, ef); t[kField].end();
  t[kFourier].begin(); field_poisson(conf, ef); t[kFourier].end();
  t[kDiag].begin(); dg->compute(conf, ef, iter); t[kDiag].end();
  t[kVx].begin(); Advection::advect_1D_vx(conf, fn, fnp1, ef, dt); t[kVx].end();
  t[kVy].begin(); Advection::advect_1D_vy(conf, fnp1, fn, ef, dt); t[kVy].end();
  t[kX].begin(); Advection::advect_1D_x(conf, fn, fnp1, 0.5 * dt); t[kX].end();
  t[kY].begin(); Advection::advect_1D_y(conf, fnp1, fn, 0.5 * dt); t[kY].end();
}

}  // namespace

int main(int argc, char **argv) {
  const char *deck = argc > 1 ? argv[1] : "data.dat";
  const bool fused = argc > 2 && std::strcmp(argv[2], "--fused") == 0;
  Config conf;
  RealView4D fn, fnp1;
  Efield *ef = nullptr;
  Diags *dg = nullptr;
  StageTimer timers[kCount];
  for (int i = 0; i < kCount; ++i) timers[i].label = kLabels[i];
  try {
    init(deck, &conf, fn, fnp1, &ef, &dg);
    int iter = 0;
    timers[kTotal].begin();
    field_rho(&conf, fn, ef);
    field_poisson(&conf, ef);
    dg->compute(&conf, ef, iter);
    if (conf.dom_.fxvx_) Advection::print_fxvx(&conf, fn, iter);
    synchronize();
    while (iter < conf.dom_.nbiter_) {
      timers[kMainLoop].begin();
      ++iter;
      if (fused) {
        timers[kStep].begin();
        vlp4d_shim::check(vlp4d_step(ef->ctx(), fn.data(), fnp1.data(), iter, nullptr), "vlp4d_step");
        fn.swap(fnp1);
        timers[kStep].end();
      } else {
        staged_step(&conf, fn, fnp1, ef, dg, timers, iter);
      }
      if (conf.dom_.fxvx_ && iter % conf.dom_.ifreq_ == 0) Advection::print_fxvx(&conf, fn, iter);
      timers[kMainLoop].end();
    }
    timers[kTotal].end();
    vlp4d_shim::check(vlp4d_check(ef->ctx()), "vlp4d_check");
    finalize(&conf, &ef, &dg);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "vlp4d_b200: %s\n", e.what());
    return 1;
  }
  for (int i = 0; i < kCount; ++i)
    if (timers[i].calls) std::printf("%s %g [s], %d calls\n", timers[i].label.c_str(), timers[i].seconds, timers[i].calls);
  return 0;
}
