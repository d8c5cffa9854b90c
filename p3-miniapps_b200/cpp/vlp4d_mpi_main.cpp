// vlp4d_mpi_b200 driver: the flow of the reference's vlp4d_mpi main()
// (miniapps/vlp4d_mpi/openmp/Vlp4d.cpp:12-62) for one process, on the C ABI.
//
//   vlp4d_mpi_b200 -f <deck> [--staged]
//
// By default each step is one vlp4d_mpi_step (four fused passes).  With
// --staged every step runs the reference's sequence (Timestep.hpp:34-97)
// through the separate entry points, timed per stage with the reference's
// timer labels (Timer.hpp:37-50; the halo fill of one process under "comm").
// Writes nrj.out (t, nrj, nrjx, nrjy, mass) and l2norm.out (t, l2norm) in
// the format of Diags::save (Diags.cpp:78-104) and prints
// "label seconds [s], calls calls".
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "../../include/vlp4d_b200.h"

namespace {

void check(int rc, const char *what) {
  if (rc != VLP4D_OK) {
    std::fprintf(stderr, "vlp4d_mpi_b200: %s: %s\n", what, vlp4d_last_error());
    std::exit(1);
  }
}

void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "vlp4d_mpi_b200: %s: %s\n", what, cudaGetErrorString(e));
    std::exit(1);
  }
}

struct StageTimer {
  std::string label;
  double seconds = 0;
  int calls = 0;
  std::chrono::steady_clock::time_point t0;
  void begin() { t0 = std::chrono::steady_clock::now(); }
  void end() {
    cuda_check(cudaDeviceSynchronize(), "synchronize");
    seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    ++calls;
  }
};

enum { kTotal, kMainLoop, kComm, kAdvec2D, kAdvec4D, kField, kDiag, kSplineXY, kSplineVV, kStep, kCount };
const char *kLabels[kCount] = {"total", "MainLoop", "comm", "advec2D", "advec4D", "field",
                               "diag", "splinecoeff_xy", "splinecoeff_vxvy", "fused_step"};

}  // namespace

int main(int argc, char **argv) {
  // Parser.hpp:16-22: -f / --file selects the deck (default data.dat).
  const char *deck = "data.dat";
  bool staged = false;
  for (int i = 1; i < argc; ++i) {
    if ((!std::strcmp(argv[i], "-f") || !std::strcmp(argv[i], "--file")) && i + 1 < argc) deck = argv[++i];
    else if (!std::strcmp(argv[i], "--staged")) staged = true;
  }
  std::printf("reading input file %s\n", deck);
  vlp4d_domain dom;
  check(vlp4d_read_deck(deck, &dom), "read_deck");
  vlp4d_ctx *ctx = nullptr;
  check(vlp4d_ctx_create(&dom, VLP4D_F64, &ctx), "ctx_create");
  const size_t bytes = vlp4d_mpi_size(ctx) * sizeof(double);
  void *fn = nullptr, *fnp1 = nullptr, *tmp = nullptr;
  cuda_check(cudaMalloc(&fn, bytes), "cudaMalloc");
  cuda_check(cudaMalloc(&fnp1, bytes), "cudaMalloc");
  if (staged) cuda_check(cudaMalloc(&tmp, bytes), "cudaMalloc");
  check(vlp4d_mpi_init_case(ctx, fn, nullptr), "init_case");

  StageTimer t[kCount];
  for (int i = 0; i < kCount; ++i) t[i].label = kLabels[i];
  const double dt = dom.dt;
  int iter = 0;
  t[kTotal].begin();
  check(vlp4d_mpi_field(ctx, fn, nullptr), "field");
  check(vlp4d_diags_compute(ctx, iter, nullptr), "diags");
  check(vlp4d_mpi_l2norm(ctx, fn, iter, nullptr), "l2norm");
  while (iter < dom.nbiter) {
    t[kMainLoop].begin();
    std::printf("iter %d\n", iter);
    ++iter;
    if (staged) {
      t[kComm].begin(); check(vlp4d_mpi_halo_fill(ctx, fn, nullptr), "halo_fill"); t[kComm].end();
      t[kSplineXY].begin(); check(vlp4d_mpi_spline_xy(ctx, fn, nullptr), "spline_xy"); t[kSplineXY].end();
      cuda_check(cudaMemcpy(fnp1, fn, bytes, cudaMemcpyDeviceToDevice), "deep_copy");
      t[kAdvec2D].begin(); check(vlp4d_mpi_advect_2d(ctx, fn, tmp, 0.5 * dt, nullptr), "advect_2d"); t[kAdvec2D].end();
      t[kField].begin(); check(vlp4d_mpi_field(ctx, fn, nullptr), "field"); t[kField].end();
      t[kDiag].begin(); check(vlp4d_diags_compute(ctx, iter, nullptr), "diags"); t[kDiag].end();
      t[kSplineVV].begin(); check(vlp4d_mpi_spline_vxvy(ctx, fnp1, nullptr), "spline_vxvy"); t[kSplineVV].end();
      t[kAdvec4D].begin(); check(vlp4d_mpi_advect_4d(ctx, fnp1, fn, dt, nullptr), "advect_4d"); t[kAdvec4D].end();
      t[kField].begin(); check(vlp4d_mpi_field(ctx, fnp1, nullptr), "field"); t[kField].end();
      t[kDiag].begin();
      check(vlp4d_diags_compute(ctx, iter, nullptr), "diags");
      check(vlp4d_mpi_l2norm(ctx, fnp1, iter, nullptr), "l2norm");
      t[kDiag].end();
    } else {
      t[kStep].begin(); check(vlp4d_mpi_step(ctx, fn, fnp1, iter, nullptr), "mpi_step"); t[kStep].end();
    }
    std::swap(fn, fnp1);  // Vlp4d.cpp:46
    t[kMainLoop].end();
  }
  t[kTotal].end();
  check(vlp4d_check(ctx), "check");

  // Diags::save (Diags.cpp:78-104).
  const int count = dom.nbiter + 1;
  std::vector<double> nrj(count), mass(count), nrjx(count), nrjy(count), l2(count);
  check(vlp4d_diags_read(ctx, nrj.data(), mass.data(), count), "diags_read");
  check(vlp4d_diags_read_ext(ctx, nrjx.data(), nrjy.data(), l2.data(), count), "diags_read_ext");
  FILE *f = std::fopen("nrj.out", "w");
  FILE *g = std::fopen("l2norm.out", "w");
  if (!f || !g) {
    std::fprintf(stderr, "vlp4d_mpi_b200: cannot write nrj.out / l2norm.out\n");
    return 1;
  }
  for (int i = 0; i < count; ++i) {
    std::fprintf(f, "%17.13e %17.13e %17.13e %17.13e %17.13e\n", i * dt, nrj[i], nrjx[i], nrjy[i], mass[i]);
    std::fprintf(g, "%17.13e %17.13e\n", i * dt, l2[i]);
  }
  std::fclose(f);
  std::fclose(g);
  for (int i = 0; i < kCount; ++i)
    if (t[i].calls) std::printf("%s %g [s], %d calls\n", t[i].label.c_str(), t[i].seconds, t[i].calls);
  cudaFree(fn);
  cudaFree(fnp1);
  cudaFree(tmp);
  vlp4d_ctx_destroy(ctx);
  return 0;
}
