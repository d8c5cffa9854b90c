// Test infrastructure (oracle only): a C-callable harness around the
// reference's own OpenMP vlp4d implementation.
//
// This file is compiled together with the UNMODIFIED reference sources
// miniapps/vlp4d/openmp/{field,efield,diags,init}.cpp and the headers they
// include (advect.hpp, timestep.hpp, lib/openmp/View.hpp, lib/OpenMP_FFT.hpp),
// read in place from the reference tree by oracle/Makefile.  Nothing here
// re-implements the algorithm: every entry point forwards to the reference
// function named in its comment, so the outputs are the reference's own.
// The two shims it needs (layout tags for <experimental/mdspan>, a subset of
// FFTW3) live in oracle/shim and oracle/fftw_subset.c.
//
// Built into oracle/_ref/libvlp4d_ref.so; loaded by oracle/oracle.py.
#include "types.hpp"
#include "config.hpp"
#include "efield.hpp"
#include "field.hpp"
#include "diags.hpp"
#include "timestep.hpp"
#include "init.hpp"

#include <omp.h>
#include <unistd.h>

#include <algorithm>
#include <climits>
#include <vector>

// miniapps/vlp4d/openmp/init.cpp:120-143 (external linkage, no header).
void initcase(Config *conf, RealView4D &fn);

namespace {
struct RefState {
  Config conf;
  RealView4D f[2];
  Efield *ef = nullptr;
  Diags *dg = nullptr;
  std::vector<Timer *> timers;
};

RealView2D *field_view(RefState *s, int which) {
  switch (which) {
    case 0: return &s->ef->rho_;
    case 1: return &s->ef->ex_;
    case 2: return &s->ef->ey_;
    default: return nullptr;
  }
}
}  // namespace

extern "C" {

int ref_max_threads() { return omp_get_max_threads(); }

// Builds the reference's Config exactly as import() does
// (miniapps/vlp4d/openmp/init.cpp:13-85) but from arguments instead of a deck,
// then allocates fn/fnp1, Efield and Diags as init() does (init.cpp:293-306).
void *ref_create(const int n[4], const double minp[4], const double maxp[4], double dt,
                 int nbiter, int idcase) {
  RefState *s = new RefState();
  Physics *phys = &s->conf.phys_;
  Domain *dom = &s->conf.dom_;
  phys->eps0_ = 1.;
  phys->echarge_ = 1.;
  phys->mass_ = 1;
  phys->omega02_ = 0;
  phys->vbeam_ = 0.;
  phys->S_ = 1;
  phys->psi_ = 0;
  for (int i = 0; i < 4; ++i) {
    dom->nxmax_[i] = (size_t)n[i];
    dom->minPhy_[i] = minp[i];
    dom->maxPhy_[i] = maxp[i];
  }
  dom->dt_ = dt;
  dom->nbiter_ = nbiter;
  dom->ifreq_ = 1;
  dom->idcase_ = idcase;
  dom->fxvx_ = 0;
  for (int i = 0; i < 4; ++i) dom->dx_[i] = (dom->maxPhy_[i] - dom->minPhy_[i]) / dom->nxmax_[i];

  s->f[0] = RealView4D("fn", dom->nxmax_);
  s->f[1] = RealView4D("fnp1", dom->nxmax_);
  s->ef = new Efield(&s->conf, {dom->nxmax_[0], dom->nxmax_[1]});
  s->dg = new Diags(&s->conf);
  defineTimers(s->timers);
  return s;
}

void ref_destroy(void *h) {
  RefState *s = (RefState *)h;
  delete s->ef;
  delete s->dg;
  freeTimers(s->timers);
  delete s;
}

void ref_set_f(void *h, int which, const double *src) {
  RefState *s = (RefState *)h;
  std::copy(src, src + s->f[which].size(), s->f[which].data());
}

void ref_get_f(void *h, int which, double *dst) {
  RefState *s = (RefState *)h;
  std::copy(s->f[which].data(), s->f[which].data() + s->f[which].size(), dst);
}

void ref_set_field(void *h, int which, const double *src) {
  RefState *s = (RefState *)h;
  RealView2D *v = field_view(s, which);
  std::copy(src, src + v->size(), v->data());
}

void ref_get_field(void *h, int which, double *dst) {
  RefState *s = (RefState *)h;
  RealView2D *v = field_view(s, which);
  std::copy(v->data(), v->data() + v->size(), dst);
}

// init.cpp:120-143 initcase -> testcaseSLD10 / testcaseTSI20 / CYL02 / CYL05.
void ref_initcase(void *h, int which) {
  RefState *s = (RefState *)h;
  initcase(&s->conf, s->f[which]);
}

// advect.hpp:112-162
void ref_advect_x(void *h, int src, int dst, double dt) {
  RefState *s = (RefState *)h;
  Advection::advect_1D_x(&s->conf, s->f[src], s->f[dst], dt);
}

// advect.hpp:164-215
void ref_advect_y(void *h, int src, int dst, double dt) {
  RefState *s = (RefState *)h;
  Advection::advect_1D_y(&s->conf, s->f[src], s->f[dst], dt);
}

// advect.hpp:217-266
void ref_advect_vx(void *h, int src, int dst, double dt) {
  RefState *s = (RefState *)h;
  Advection::advect_1D_vx(&s->conf, s->f[src], s->f[dst], s->ef, dt);
}

// advect.hpp:269-317
void ref_advect_vy(void *h, int src, int dst, double dt) {
  RefState *s = (RefState *)h;
  Advection::advect_1D_vy(&s->conf, s->f[src], s->f[dst], s->ef, dt);
}

// field.cpp:5-29
void ref_field_rho(void *h, int src) {
  RefState *s = (RefState *)h;
  field_rho(&s->conf, s->f[src], s->ef);
}

// field.cpp:31-92 (-> efield.cpp:50-104)
void ref_field_poisson(void *h) {
  RefState *s = (RefState *)h;
  field_poisson(&s->conf, s->ef);
}

// diags.cpp:13-41
void ref_diags_compute(void *h, int iter) {
  RefState *s = (RefState *)h;
  s->dg->compute(&s->conf, s->ef, iter);
}

// diags.cpp:43-53 writes "nrj.out" into the working directory; this runs it
// with `dir` as the working directory and restores the previous one.
int ref_diags_save(void *h, const char *dir) {
  RefState *s = (RefState *)h;
  char prev[PATH_MAX];
  if (!getcwd(prev, sizeof(prev))) return -1;
  if (chdir(dir) != 0) return -2;
  s->dg->save(&s->conf);
  return chdir(prev) == 0 ? 0 : -3;
}

// timestep.hpp:11-55; f[0] holds the state before and after, f[1] is scratch.
void ref_onetimestep(void *h, int iter) {
  RefState *s = (RefState *)h;
  onetimestep(&s->conf, s->f[0], s->f[1], s->ef, s->dg, s->timers, iter);
}

// The body of main() in miniapps/vlp4d/openmp/vlp4d.cpp:58-74 without deck
// parsing or printing: initial rho/poisson/diag, then `nsteps` time steps.
void ref_run(void *h, int nsteps) {
  RefState *s = (RefState *)h;
  int iter = 0;
  s->timers[Total]->begin();
  field_rho(&s->conf, s->f[0], s->ef);
  field_poisson(&s->conf, s->ef);
  s->dg->compute(&s->conf, s->ef, iter);
  while (iter < nsteps) {
    s->timers[MainLoop]->begin();
    iter++;
    onetimestep(&s->conf, s->f[0], s->f[1], s->ef, s->dg, s->timers, iter);
    s->timers[MainLoop]->end();
  }
  s->timers[Total]->end();
}

// Timer idx follows TimerEnum in miniapps/vlp4d/timer.hpp:40-49.
double ref_timer_seconds(void *h, int idx, int *calls) {
  RefState *s = (RefState *)h;
  if (calls) *calls = s->timers[idx]->calls();
  return s->timers[idx]->seconds();
}

void ref_reset_timers(void *h) {
  RefState *s = (RefState *)h;
  resetTimers(s->timers);
}

// The reference's 2D real FFT (lib/OpenMP_FFT.hpp:106-142) on a layout_left
// (nx1, nx2, batch) array; `out` receives (nx1/2+1, nx2, batch) complex
// values as interleaved (re, im) pairs.
void ref_rfft2(int nx1, int nx2, int batch, double *in, double *out) {
  Impl::FFT<double, stdex::layout_left> fft(nx1, nx2, batch);
  fft.rfft2(in, reinterpret_cast<Impl::complex<double> *>(out));
}

void ref_irfft2(int nx1, int nx2, int batch, double *in, double *out) {
  Impl::FFT<double, stdex::layout_left> fft(nx1, nx2, batch);
  fft.irfft2(reinterpret_cast<Impl::complex<double> *>(in), out);
}

}  // extern "C"
