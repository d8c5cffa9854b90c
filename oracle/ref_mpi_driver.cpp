// Test infrastructure (oracle only): a C-callable harness around the
// reference's own OpenMP vlp4d_mpi implementation, run as one process.
//
// This file is compiled together with the UNMODIFIED reference sources
// miniapps/vlp4d_mpi/openmp/{Communication,Diags,Efield,Field,Init}.cpp and
// the headers they include (Timestep.hpp, Spline.hpp, Advection.hpp,
// Communication.hpp, lib/openmp/View.hpp, lib/OpenMP_FFT.hpp,
// lib/OpenMP_Transpose.hpp), read in place from the reference tree by
// oracle/Makefile.  Every entry point forwards to the reference function
// named in its comment, so the outputs are the reference's own.  The shims
// it needs are oracle/shim/mpi.h (one-process MPI), oracle/shim/fftw3.h with
// oracle/fftw_subset.c, and the mdspan layout tags.
//
// Arrays are the reference's halo-extended views: extents n[d] + 6, first
// index -3 in every dimension (HALO_PTS = 3, Config.hpp:7), layout_left.
//
// Built into oracle/_ref/libvlp4d_mpi_ref.so; loaded by oracle/oracle.py.
#include "Types.hpp"
#include "Config.hpp"
#include "Communication.hpp"
#include "Efield.hpp"
#include "Diags.hpp"
#include "Field.hpp"
#include "Init.hpp"
#include "Timestep.hpp"

#include <omp.h>
#include <unistd.h>

#include <algorithm>
#include <climits>
#include <vector>

// miniapps/vlp4d_mpi/openmp/Init.cpp:126-148 and 279-322 (external
// linkage, no header).
void initcase(Config *conf, RealView4D &fn);
void testcase_ptest_init(Config *conf, Distrib &comm, RealView4D &halo_fn);
void testcase_ptest_check(Config *conf, Distrib &comm, RealView4D &halo_fn);

namespace {
struct RefMpiState {
  Config conf;
  Distrib *comm = nullptr;
  RealView4D f[2];
  Efield *ef = nullptr;
  Diags *dg = nullptr;
  Impl::Transpose<float64, default_layout> *transpose = nullptr;
  std::vector<Timer *> timers;
};

RealView2D *field_view(RefMpiState *s, int which) {
  switch (which) {
    case 0: return &s->ef->rho_;
    case 1: return &s->ef->ex_;
    case 2: return &s->ef->ey_;
    case 3: return &s->ef->phi_;
    default: return nullptr;
  }
}
}  // namespace

extern "C" {

int refm_max_threads() { return omp_get_max_threads(); }

int refm_halo_pts() { return HALO_PTS; }

// Builds the Config exactly as import() does (Init.cpp:12-90) from arguments
// instead of a deck, then follows init() (Init.cpp:324-373): decomposition
// over the one process, halo views, neighbour lists and halo bookkeeping,
// the halo self-test exchange, Efield, Diags, the transpose, and the initial
// condition of case `idcase` in fn (views index 0 = fn, 1 = fnp1).
void *refm_create(const int n[4], const double minp[4], const double maxp[4], double dt, int nbiter,
                  int idcase) {
  RefMpiState *s = new RefMpiState();
  int argc = 1;
  static char arg0[] = "vlp4d_mpi";
  char *argv_store[] = {arg0, nullptr};
  char **argv = argv_store;
  s->comm = new Distrib(argc, argv);
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
  dom->fxvx_ = 0;
  dom->idcase_ = idcase;
  for (int i = 0; i < 4; ++i) dom->dx_[i] = (dom->maxPhy_[i] - dom->minPhy_[i]) / dom->nxmax_[i];

  defineTimers(s->timers);
  Distrib &comm = *s->comm;
  comm.createDecomposition(&s->conf);
  Urbnode *mynode = comm.node();
  shape_nd<DIMENSION> shape_halo;
  range_nd<DIMENSION> nxmin_halo;
  for (int i = 0; i < DIMENSION; i++) nxmin_halo[i] = mynode->xmin_[i] - HALO_PTS;
  for (int i = 0; i < DIMENSION; i++) shape_halo[i] = mynode->xmax_[i] - mynode->xmin_[i] + 2 * HALO_PTS + 1;
  const int nx = shape_halo[0], ny = shape_halo[1], nvx = shape_halo[2], nvy = shape_halo[3];
  s->f[0] = RealView4D("fn", shape_halo, nxmin_halo);
  s->f[1] = RealView4D("fnp1", shape_halo, nxmin_halo);
  s->f[0].fill(0);
  s->f[1].fill(0);
  comm.neighboursList(&s->conf, s->f[0]);
  comm.bookHalo(&s->conf);
  testcase_ptest_init(&s->conf, comm, s->f[0]);
  comm.exchangeHalo(&s->conf, s->f[0], s->timers);
  testcase_ptest_check(&s->conf, comm, s->f[0]);
  resetTimers(s->timers);
  s->ef = new Efield(&s->conf, {dom->nxmax_[0], dom->nxmax_[1]});
  s->dg = new Diags(&s->conf);
  s->transpose = new Impl::Transpose<float64, default_layout>(nx * ny, nvx * nvy);
  s->f[0] = RealView4D("fn", shape_halo, nxmin_halo);
  s->f[0].fill(0);
  initcase(&s->conf, s->f[0]);
  return s;
}

void refm_destroy(void *h) {
  RefMpiState *s = (RefMpiState *)h;
  delete s->ef;
  delete s->dg;
  delete s->transpose;
  s->comm->cleanup();
  delete s->comm;
  freeTimers(s->timers);
  delete s;
}

// Whole halo-extended arrays ((n+6)^4 doubles, layout_left).
void refm_set_f(void *h, int which, const double *src) {
  RefMpiState *s = (RefMpiState *)h;
  std::copy(src, src + s->f[which].size(), s->f[which].data());
}

void refm_get_f(void *h, int which, double *dst) {
  RefMpiState *s = (RefMpiState *)h;
  std::copy(s->f[which].data(), s->f[which].data() + s->f[which].size(), dst);
}

void refm_set_field(void *h, int which, const double *src) {
  RefMpiState *s = (RefMpiState *)h;
  RealView2D *v = field_view(s, which);
  std::copy(src, src + v->size(), v->data());
}

void refm_get_field(void *h, int which, double *dst) {
  RefMpiState *s = (RefMpiState *)h;
  RealView2D *v = field_view(s, which);
  std::copy(v->data(), v->data() + v->size(), dst);
}

// Init.cpp:126-148 initcase (SLD10 / TSI20 / CYL02 / CYL05) on the interior.
void refm_initcase(void *h, int which) {
  RefMpiState *s = (RefMpiState *)h;
  initcase(&s->conf, s->f[which]);
}

// Communication.cpp:541-570: halo exchange with the spline boundary sums
// (Communication.hpp:756-896); one process: local copies only.
void refm_exchange_halo(void *h, int which) {
  RefMpiState *s = (RefMpiState *)h;
  s->comm->exchangeHalo(&s->conf, s->f[which], s->timers);
}

// Spline.hpp:384-426 / 429-469: cubic spline coefficients along x, y
// (in place) / along vx, vy (through the transpose).
void refm_spline_xy(void *h, int which) {
  RefMpiState *s = (RefMpiState *)h;
  Spline::computeCoeff_xy(&s->conf, s->transpose, s->f[which]);
}

void refm_spline_vxvy(void *h, int which) {
  RefMpiState *s = (RefMpiState *)h;
  Spline::computeCoeff_vxvy(&s->conf, s->transpose, s->f[which]);
}

// Advection.hpp:299-406: 2D x, y advection of view `which` by dt (spline
// coefficients in, values out on the interior).
void refm_advect_2d(void *h, int which, double dt) {
  RefMpiState *s = (RefMpiState *)h;
  Advection::advect_2D_xy(&s->conf, s->f[which], dt);
}

// Advection.hpp:409-498: 4D advection advect_4D(conf, ef, fn = f[dst],
// tmp_fn = f[src], dt): the coefficients in f[dst] are copied to f[src] and
// f[dst]'s interior receives the interpolated values.
void refm_advect_4d(void *h, int dst, int src, double dt) {
  RefMpiState *s = (RefMpiState *)h;
  Advection::advect_4D(&s->conf, s->ef, s->f[dst], s->f[src], dt);
}

// Field.cpp:5-55, 57-69, 71-132: rho of view `which`, the (one-process)
// reduction and the Poisson solve.
void refm_field(void *h, int which) {
  RefMpiState *s = (RefMpiState *)h;
  field_rho(&s->conf, s->f[which], s->ef);
  field_reduce(&s->conf, s->ef);
  field_poisson(&s->conf, s->ef);
}

// Diags.cpp:16-48 and 50-76.
void refm_diags(void *h, int iter) {
  RefMpiState *s = (RefMpiState *)h;
  s->dg->compute(&s->conf, s->ef, iter);
}

void refm_l2norm(void *h, int which, int iter) {
  RefMpiState *s = (RefMpiState *)h;
  s->dg->computeL2norm(&s->conf, s->f[which], iter);
}

// Diags.cpp:78-104 writes nrj.out and l2norm.out into the working directory;
// this runs it with `dir` as the working directory and restores the old one.
int refm_diags_save(void *h, const char *dir) {
  RefMpiState *s = (RefMpiState *)h;
  char prev[PATH_MAX];
  if (!getcwd(prev, sizeof(prev))) return -1;
  if (chdir(dir) != 0) return -2;
  s->dg->save(&s->conf, *s->comm);
  return chdir(prev) == 0 ? 0 : -3;
}

// Timestep.hpp:34-97 followed by the swap of Vlp4d.cpp:46: f[0] holds the
// state before and after the step.
void refm_onetimestep(void *h, int iter) {
  RefMpiState *s = (RefMpiState *)h;
  onetimestep(&s->conf, *s->comm, s->f[0], s->f[1], s->ef, s->dg, s->transpose, s->timers, iter);
  s->f[0].swap(s->f[1]);
}

// The body of main() in miniapps/vlp4d_mpi/openmp/Vlp4d.cpp:30-49 without
// deck parsing or printing: initial field and diagnostics, then `nsteps`
// time steps.
void refm_run(void *h, int nsteps) {
  RefMpiState *s = (RefMpiState *)h;
  int iter = 0;
  s->timers[Total]->begin();
  field_rho(&s->conf, s->f[0], s->ef);
  field_reduce(&s->conf, s->ef);
  field_poisson(&s->conf, s->ef);
  s->dg->compute(&s->conf, s->ef, iter);
  s->dg->computeL2norm(&s->conf, s->f[0], iter);
  while (iter < nsteps) {
    s->timers[MainLoop]->begin();
    iter++;
    onetimestep(&s->conf, *s->comm, s->f[0], s->f[1], s->ef, s->dg, s->transpose, s->timers, iter);
    s->f[0].swap(s->f[1]);
    s->timers[MainLoop]->end();
  }
  s->timers[Total]->end();
}

// Timer idx follows TimerEnum in miniapps/vlp4d_mpi/Timer.hpp:37-50.
double refm_timer_seconds(void *h, int idx, int *calls) {
  RefMpiState *s = (RefMpiState *)h;
  if (calls) *calls = s->timers[idx]->calls();
  return s->timers[idx]->seconds();
}

void refm_reset_timers(void *h) {
  RefMpiState *s = (RefMpiState *)h;
  resetTimers(s->timers);
}

}  // extern "C"
