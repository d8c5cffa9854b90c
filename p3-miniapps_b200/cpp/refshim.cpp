// Reference-facing C++ layer: implementations of the reference's L3
// functions (Efield, Diags, field_rho, field_poisson, Advection::*, init,
// finalize) on top of the C ABI of libvlp4d_b200.  Each forwards to one C
// entry point; the reference function it stands in for is cited.
#include <cstdio>
#include <mutex>
#include <unordered_map>

#include "refshim/advection.hpp"
#include "refshim/config.hpp"
#include "refshim/diags.hpp"
#include "refshim/efield.hpp"
#include "refshim/field.hpp"
#include "refshim/init.hpp"

using vlp4d_shim::check;

namespace vlp4d_shim {
namespace {
std::mutex g_mu;
std::unordered_map<const Config *, vlp4d_ctx *> g_ctx;
}  // namespace

vlp4d_ctx *context_of(const Config *conf) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_ctx.find(conf);
  if (it == g_ctx.end()) throw std::runtime_error("no Efield has been created for this Config");
  return it->second;
}
}  // namespace vlp4d_shim

// efield.cpp:5-37: fields, FFT plans (and here also the diagnostic history).
Efield::Efield(Config *conf, shape_nd<2> dim) : conf_(conf) {
  const vlp4d_domain d = vlp4d_shim::to_domain(conf);
  if (d.nxmax[0] != dim[0] || d.nxmax[1] != dim[1]) throw std::invalid_argument("Efield: dim differs from Config");
  check(vlp4d_ctx_create(&d, VLP4D_F64, &ctx_), "vlp4d_ctx_create");
  double *p = nullptr;
  check(vlp4d_field_ptr(ctx_, VLP4D_FIELD_RHO, &p), "vlp4d_field_ptr");
  rho_ = RealView2D::wrap("rho", p, dim);
  check(vlp4d_field_ptr(ctx_, VLP4D_FIELD_EX, &p), "vlp4d_field_ptr");
  ex_ = RealView2D::wrap("ex", p, dim);
  check(vlp4d_field_ptr(ctx_, VLP4D_FIELD_EY, &p), "vlp4d_field_ptr");
  ey_ = RealView2D::wrap("ey", p, dim);
  phi_ = RealView2D("phi", dim);
  std::lock_guard<std::mutex> lk(vlp4d_shim::g_mu);
  vlp4d_shim::g_ctx[conf] = ctx_;
}

Efield::~Efield() {
  {
    std::lock_guard<std::mutex> lk(vlp4d_shim::g_mu);
    vlp4d_shim::g_ctx.erase(conf_);
  }
  vlp4d_ctx_destroy(ctx_);
}

// efield.cpp:43-105 (the caller has already applied rho -= 1 where the
// reference's field_poisson does).
void Efield::solve_poisson_fftw(float64, float64) { check(vlp4d_field_poisson(ctx_, nullptr), "field_poisson"); }

// diags.cpp:6-11: the history is allocated with the Efield's context.
Diags::Diags(Config *) {}
Diags::~Diags() {}

// diags.cpp:13-55.
void Diags::compute(Config *, Efield *ef, int iter) {
  check(vlp4d_diags_compute(ef->ctx(), iter, nullptr), "diags_compute");
}

// diags.cpp:57-68.
void Diags::save(Config *conf) { check(vlp4d_diags_save(vlp4d_shim::context_of(conf), "nrj.out"), "diags_save"); }

// field.cpp:6-32.
void field_rho(Config *, RealView4D &fn, Efield *ef) { check(vlp4d_field_rho(ef->ctx(), fn.data(), nullptr), "field_rho"); }

// field.cpp:34-82 (the case switch, rho -= 1 and the solve).
void field_poisson(Config *, Efield *ef) { check(vlp4d_field_poisson(ef->ctx(), nullptr), "field_poisson"); }

namespace Advection {
// advection.hpp:336-347
void advect_1D_x(Config *conf, const RealView4D &fn, RealView4D &fnp1, float64 dt) {
  check(vlp4d_advect_x(vlp4d_shim::context_of(conf), fn.data(), fnp1.data(), dt, nullptr), "advect_1D_x");
}
// advection.hpp:349-360
void advect_1D_y(Config *conf, const RealView4D &fn, RealView4D &fnp1, float64 dt) {
  check(vlp4d_advect_y(vlp4d_shim::context_of(conf), fn.data(), fnp1.data(), dt, nullptr), "advect_1D_y");
}
// advection.hpp:362-373
void advect_1D_vx(Config *, const RealView4D &fn, RealView4D &fnp1, Efield *ef, float64 dt) {
  check(vlp4d_advect_vx(ef->ctx(), fn.data(), fnp1.data(), dt, nullptr), "advect_1D_vx");
}
// advection.hpp:375-386
void advect_1D_vy(Config *, const RealView4D &fn, RealView4D &fnp1, Efield *ef, float64 dt) {
  check(vlp4d_advect_vy(ef->ctx(), fn.data(), fnp1.data(), dt, nullptr), "advect_1D_vy");
}
// advection.hpp:388-411
void print_fxvx(Config *conf, RealView4D &fn, int iter) {
  char filename[128];
  printf("print_fxvx %d\n", iter);
  snprintf(filename, sizeof(filename), "data/vlp4d/fxvx_it%06d.csv", iter);
  check(vlp4d_print_fxvx(vlp4d_shim::context_of(conf), fn.data(), filename), "print_fxvx");
}
}  // namespace Advection

// init.cpp:287-305: parse the deck, allocate f, Efield and Diags, fill the
// initial condition of the deck's test case on the device.
void init(const char *file, Config *conf, RealView4D &fn, RealView4D &fnp1, Efield **ef, Diags **dg) {
  vlp4d_domain d;
  check(vlp4d_read_deck(file, &d), "read deck");
  Domain *dom = &conf->dom_;
  Physics *phys = &conf->phys_;
  phys->eps0_ = 1.;
  phys->echarge_ = 1.;
  phys->mass_ = 1;
  phys->omega02_ = 0;
  phys->vbeam_ = 0.;
  phys->S_ = 1;
  phys->psi_ = 0;
  for (size_t i = 0; i < DIMENSION; ++i) {
    dom->nxmax_[i] = d.nxmax[i];
    dom->minPhy_[i] = d.min_phy[i];
    dom->maxPhy_[i] = d.max_phy[i];
    dom->dx_[i] = (dom->maxPhy_[i] - dom->minPhy_[i]) / dom->nxmax_[i];
  }
  dom->dt_ = d.dt;
  dom->nbiter_ = d.nbiter;
  dom->ifreq_ = d.ifreq;
  dom->idcase_ = d.idcase;
  dom->fxvx_ = d.fxvx;
  printf("** vlp4d on B200: %d x %d x %d x %d, case %d, dt %lf, %d steps\n", dom->nxmax_[0], dom->nxmax_[1],
         dom->nxmax_[2], dom->nxmax_[3], dom->idcase_, dom->dt_, dom->nbiter_);
  fn = RealView4D("fn", dom->nxmax_[0], dom->nxmax_[1], dom->nxmax_[2], dom->nxmax_[3]);
  fnp1 = RealView4D("fnp1", dom->nxmax_[0], dom->nxmax_[1], dom->nxmax_[2], dom->nxmax_[3]);
  *ef = new Efield(conf, {dom->nxmax_[0], dom->nxmax_[1]});
  *dg = new Diags(conf);
  // init.cpp:118-141 aborts on an unknown case; vlp4d_init_case rejects it.
  check(vlp4d_init_case((*ef)->ctx(), fn.data(), dom->idcase_, 0.05, 0.5, 2.4, nullptr), "initcase");
}

// init.cpp:307-313.
void finalize(Config *conf, Efield **ef, Diags **dg) {
  (*dg)->save(conf);
  delete *ef;
  delete *dg;
  *ef = nullptr;
  *dg = nullptr;
}
