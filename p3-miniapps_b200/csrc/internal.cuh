// Internal declarations shared by the translation units of libvlp4d_b200.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/vlp4d_b200.h"
#include "lagrange.cuh"

namespace vlp4d {

constexpr int kNumSMs = 148;  // B200; the launchers read the real count from the device

// Thread-local last error message (vlp4d_last_error).
void set_error(const std::string &msg);

// Process-wide count of this library's own kernel launches (cuFFT's are not
// included), read by vlp4d_kernel_launches().
void count_launch();

#define VLP4D_CUDA_TRY(expr)                                                                   \
  do {                                                                                         \
    cudaError_t _e = (expr);                                                                   \
    if (_e != cudaSuccess) {                                                                   \
      ::vlp4d::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));                  \
      return VLP4D_ERR_CUDA;                                                                   \
    }                                                                                          \
  } while (0)

#define VLP4D_CUFFT_TRY(expr)                                                                  \
  do {                                                                                         \
    cufftResult _r = (expr);                                                                   \
    if (_r != CUFFT_SUCCESS) {                                                                 \
      ::vlp4d::set_error(std::string(#expr) + ": cufft error " + std::to_string((int)_r));     \
      return VLP4D_ERR_CUDA;                                                                   \
    }                                                                                          \
  } while (0)

#define VLP4D_LAUNCH_CHECK()                                                                   \
  do {                                                                                         \
    ::vlp4d::count_launch();                                                                   \
    cudaError_t _e = cudaGetLastError();                                                       \
    if (_e != cudaSuccess) {                                                                   \
      ::vlp4d::set_error(std::string("kernel launch: ") + cudaGetErrorString(_e));             \
      return VLP4D_ERR_CUDA;                                                                   \
    }                                                                                          \
  } while (0)

// Geometry of one run, in the reference's Domain terms.
struct Grid {
  int n[4];          // nx, ny, nvx, nvy
  double minp[4], maxp[4], dx[4];
  __host__ __device__ long long nxy() const { return (long long)n[0] * n[1]; }
  __host__ __device__ long long nv() const { return (long long)n[2] * n[3]; }
  __host__ __device__ long long cells() const { return nxy() * nv(); }
};

// Device-side line stencil tables, one entry per swept line.
//   m[line] : tap offset, w[6*line + k] : FP64 weights,
//   wf[6*line + j] : FP32 difference weights (stencil.cuh), j < 5.
struct StencilTable {
  int *m = nullptr;
  // vy tables built for the v-slab pass: per chunk of span_C consecutive
  // lines the smallest and largest signed offset (span_C = 0: none; the
  // pass then computes them).
  int2 *span = nullptr;
  int span_C = 0;
  double *w = nullptr;
  float *wf = nullptr;
  int lines = 0;
  double dt = 0.0;  // the dt the table was built for (host-built tables only)
  bool valid = false;
  unsigned long long stamp = 0;  // last use, for slot replacement
};

}  // namespace vlp4d

struct vlp4d_ctx {
  vlp4d::Grid g;
  vlp4d_domain dom;
  int dtype;           // VLP4D_F64 / VLP4D_F32
  int device;
  int num_sms;
  size_t elem;         // sizeof element of f

  // Efield equivalents (FP64, nx*ny).
  double *rho = nullptr, *ex = nullptr, *ey = nullptr;
  // Spectral work arrays ((nx/2+1)*ny complex).
  cufftDoubleComplex *rho_hat = nullptr, *ex_hat = nullptr, *ey_hat = nullptr;
  cufftHandle plan_fwd = 0, plan_bwd = 0;
  // The three inverse transforms of the field solve (phi, ex, ey) as one
  // batched plan: rho/ex/ey and their spectra are slices of one allocation
  // each, at the strides below.
  cufftHandle plan_bwd3 = 0;
  size_t fstride = 0, hstride = 0;
  bool plans = false;
  // The cluster field solve (k_field_cluster) instead of the cuFFT plans:
  // -1 not yet decided, 0 no (shape, VLP4D_FIELD=cufft, or no cluster
  // fits), else the cluster size (8 or 16).
  int field_cluster = -1;
  int field_cluster_t = -1;  // the same for the transposed solve (reverse mode)

  // Diagnostics history (nbiter+1 entries each) and the reduction scratch.
  double *nrj = nullptr, *mass = nullptr;
  // The vlp4d_mpi diagnostics (miniapps/vlp4d_mpi/thrust/Diags.cpp:17-92):
  // per-component field energies and the L2 norm of f, one slot per iteration.
  double *nrjx = nullptr, *nrjy = nullptr, *l2norm = nullptr;
  // L2-norm partial sums (Kahan pairs, one per block of k_l2_partial).
  double *l2_part = nullptr;
  int l2_blocks = 0;
  int hist_len = 0;

  // Moment partials: rho_part_groups x nxy FP64.  The generic reduction
  // uses rho_groups of them, the fused x/y pass up to rho_part_groups.
  double *rho_part = nullptr;
  int rho_groups = 0;
  int rho_part_groups = 0;
  // VLP4D_XYXY at creation: -1 unset, 0 never join x/y half steps across
  // steps, 1 always (when the kernel fits the shape).
  int xyxy_mode = -1;

  // Kernel selection, read from VLP4D_KERNELS at context creation:
  // unset = fused kernels where the shape allows, generic otherwise;
  // "generic" = generic per-cell kernels only; "fused" = fused kernels only
  // (an unsupported shape is an error instead of a silent fallback).
  bool fused = true;
  bool fused_only = false;
  // Error word: bit 1 set by a kernel whose bounded wait for an asynchronous
  // copy ran out, bit 2 by a vlp4d_mpi advection whose foot left the
  // interpolation range.
  int *d_err = nullptr;
  // Per column chunk (min, max) signed vy offset for the fused v pass.
  int2 *vspan = nullptr;
  int vspan_cap = 0;

  // Stencil tables: x/y lines for the two dt values of a Strang step (built
  // on the host and uploaded once), v lines rebuilt from E on the device.
  vlp4d::StencilTable tab_x[2], tab_y[2];
  vlp4d::StencilTable tab_vx, tab_vy;
  // Two x (y) shifts by the same dt composed into one 11-tap stencil, for
  // the x/y/x/y pass: m = 2*m1 mod n, w = w1 * w1 (convolution).
  vlp4d::StencilTable tab_x11, tab_y11;
  unsigned long long table_clock = 0;

  // Pinned host staging for vlp4d_run's per-step diagnostic read-back.
  double *h_diag = nullptr;

  // Per-block (sum, compensation) pairs of the vlp4d_mpi L2 norm and 4D
  // pass (mpi.cu), mpi_part_cap pairs.
  double *mpi_part = nullptr;
  int mpi_part_cap = 0;

  // vy-slab contexts (vlp4d_ctx_create_slab): this context owns the global
  // vy planes [ivy0, ivy0 + g.n[3]) of a run with nvy_glob planes.  g holds
  // the local extents (g.n[3] = owned planes) with the GLOBAL vy geometry
  // (minp/maxp/dx[3]), so tables and coordinates use global indices.  An f
  // buffer of a slab context holds `halo` planes on each side of the owned
  // ones: nx*ny*nvx*(g.n[3] + 2*halo) elements, owned planes from plane
  // `halo` on.  For ordinary contexts slab = false, ivy0 = halo = 0 and
  // nvy_glob = g.n[3].
  bool slab = false;
  int ivy0 = 0, halo = 0, nvy_glob = 0;

  // The energy/mass diagnostic of a time step reads only the solved field
  // and nothing on the step's critical path reads its result, so the time
  // loops run it on this side stream (forked after the field solve, joined
  // before rho is next written), overlapping the v-table build and the vx/vy
  // pass.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

namespace vlp4d {

// Error-word bits (vlp4d_check): a bounded wait ran out; a vlp4d_mpi foot
// left its interpolation range; a slab's vy sweep needed planes beyond its
// halo.
constexpr int kErrTimeout = 1, kErrMpiRange = 2, kErrSlabHalo = 4;

// Planes of one (ivx, ivy) plane times nvx: elements between consecutive ivy.
inline size_t vy_plane_elems(const vlp4d_ctx *c) { return (size_t)c->g.nxy() * c->g.n[2]; }
// The owned planes of an f buffer (the buffer itself for ordinary contexts).
inline const void *owned_planes(const vlp4d_ctx *c, const void *f) {
  return static_cast<const char *>(f) + (size_t)c->halo * vy_plane_elems(c) * c->elem;
}
inline void *owned_planes(const vlp4d_ctx *c, void *f) {
  return static_cast<char *>(f) + (size_t)c->halo * vy_plane_elems(c) * c->elem;
}

// advect.cu
int alloc_table(StencilTable &t, int lines, int taps = 6);
// The span buffer of a vy table for chunks of C lines (lines / C entries).
int alloc_span(StencilTable &t, int C);
// Columns per chunk of the v-slab pass of this context (0: the pass does
// not run on this shape).
int vslab_chunk_cols(const vlp4d_ctx *c);
// Signed form of a tap offset m in [0, n): the shift in cells, in (-n/2, n/2].
__host__ __device__ __forceinline__ int signed_offset(int m, int n) { return m > n / 2 ? m - n : m; }
// Per chunk of C consecutive lines (C divides 32; lines and lanes
// consecutive, chunks aligned to warps): lane `line % C == 0` stores the
// smallest and largest o of its chunk.  Every lane of the warp calls it;
// `on` false for lanes past the last line.
__device__ __forceinline__ void chunk_span(bool on, int o, int line, int C, int2 *span) {
  int lo = on ? o : (1 << 30), hi = on ? o : -(1 << 30);
  for (int d = C >> 1; d > 0; d >>= 1) {
    const int l2 = __shfl_xor_sync(0xffffffffu, lo, d), h2 = __shfl_xor_sync(0xffffffffu, hi, d);
    lo = l2 < lo ? l2 : lo;
    hi = h2 > hi ? h2 : hi;
  }
  if (on && line % C == 0) span[line / C] = make_int2(lo, hi);
}
void free_table(StencilTable &t);
int ensure_xy_table(vlp4d_ctx *c, int dim, double dt, StencilTable **out, cudaStream_t s);
// The composed 11-tap table of two x (dim 0) or y (dim 1) shifts by dt:
// per line m and 11 FP64 weights; for FP32, 10 difference weights about tap 5.
int ensure_xy11_table(vlp4d_ctx *c, int dim, double dt, StencilTable **out, cudaStream_t s);
// The 11-tap line of two applications of the 6-tap line st on n points:
// offset 2m mod n, FP64 weights W = w * w, FP32 difference weights u.
void line11(const LineStencil &st, int n, int *m, double W[11], float u[10]);
// An 11-tap x (dim 0) or y (dim 1) table for two shifts by dt, of the
// transposed lines when `transposed` (the reverse mode's joined pass).
int build_xy11_table(vlp4d_ctx *c, int dim, double dt, bool transposed, StencilTable &t, cudaStream_t s);
int build_v_tables(vlp4d_ctx *c, double dt, bool vx, bool vy, cudaStream_t s);
int launch_advect_generic(vlp4d_ctx *c, int dim, const void *fn, void *fnp1, const StencilTable *t,
                          cudaStream_t s);
int launch_advect_pair_generic(vlp4d_ctx *c, bool v, const void *fn, void *fnp1, const StencilTable *ta,
                               const StencilTable *tb, cudaStream_t s);
// Slab contexts: the vy sweep (with the vx sweep first when tvx is given) of
// the owned planes from an input buffer whose halo planes are filled; one
// thread per output cell, any shape.  fn_ext is the whole input buffer,
// fnp1_owned the owned planes of the output.
int launch_vy_slab_generic(vlp4d_ctx *c, const void *fn_ext, void *fnp1_owned, const StencilTable *tvx,
                           const StencilTable *tvy, cudaStream_t s);
// advect_plane.cu / advect_vslab.cu: VLP4D_ERR_UNSUPPORTED (nothing
// launched) when the shape or buffers do not fit; callers then use the
// generic kernels.
int launch_advect_xy(vlp4d_ctx *c, const void *fn, void *fnp1, const StencilTable *tx,
                     const StencilTable *ty, bool do_x, bool do_y, bool with_rho, cudaStream_t s);
int launch_advect_vxvy(vlp4d_ctx *c, const void *fn, void *fnp1, bool do_vx, bool do_vy, cudaStream_t s);
// The same pass with explicit v tables (the reverse mode passes transposed
// ones) and an optional per-column term: out += bias_scale * bias[ix + nx*iy].
int launch_advect_vxvy_tables(vlp4d_ctx *c, const void *fn, void *fnp1, const StencilTable *tvx,
                              const StencilTable *tvy, cudaStream_t s, const double *bias = nullptr,
                              double bias_scale = 0.0);
int launch_advect_xyxy(vlp4d_ctx *c, const void *fn, void *fnp1, const StencilTable *tx, const StencilTable *ty,
                       cudaStream_t s);
// Whether the FP64 form of the joined pass (k_plane_xyxy64, row widths a
// warp holds whole) runs for this context.
bool xyxy64_available(const vlp4d_ctx *c);
// The same pass with explicit 11-tap tables.  with_rho false leaves the
// context's rho alone (the kernels without a moment-free form still write
// their partial moments into the context's scratch).
int launch_advect_xyxy_tables(vlp4d_ctx *c, const void *fn, void *fnp1, const StencilTable *x11,
                              const StencilTable *y11, bool with_rho, cudaStream_t s);

// api.cu: one Strang step f_in -> f_out through scratch (diagnostic slot
// `iter`, none when negative); x/y and vx/vy passes with explicit tables,
// fused kernels first, generic ones when the fused kernels decline.
int step_impl(vlp4d_ctx *ctx, const void *f_in, void *f_out, void *scratch, int iter, cudaStream_t s);
int advect_xy_moment(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, cudaStream_t s);
int advect_xy_any(vlp4d_ctx *ctx, const void *fn, void *fnp1, const StencilTable *tx, const StencilTable *ty,
                  cudaStream_t s);
int advect_vxvy_any(vlp4d_ctx *ctx, const void *fn, void *fnp1, const StencilTable *tvx, const StencilTable *tvy,
                    cudaStream_t s);
// Records msg as the calling thread's last error and returns code.
int fail_msg(int code, const std::string &msg);
// Whether time loops join the x/y half steps of consecutive steps into one
// k_plane_xyxy pass (FP32 by default; VLP4D_XYXY overrides).
bool xyxy_join(const vlp4d_ctx *ctx);

// field.cu
int launch_field_rho(vlp4d_ctx *c, const void *fn, cudaStream_t s);
int launch_rho_finish(vlp4d_ctx *c, int groups, cudaStream_t s);
int launch_field_poisson(vlp4d_ctx *c, cudaStream_t s);
// The cluster field solve (field_cluster.cu): whether it serves this
// context, and its launch (rho - offset -> phi in rho, ex, ey).
bool field_cluster_available(vlp4d_ctx *c);
int launch_field_cluster(vlp4d_ctx *c, double offset, cudaStream_t s);
// The transposed solve lam_rho = D^T (gex, gey) from the impulse-response
// spectra (half-spectrum layout of the forward D2Z).
bool field_cluster_t_available(vlp4d_ctx *c);
int launch_field_transpose_cluster(vlp4d_ctx *c, const double *gex, const double *gey, const void *hx_hat,
                                   const void *hy_hat, double *lam_rho, cudaStream_t s);
int launch_diags(vlp4d_ctx *c, int iter, cudaStream_t s);
// launch_diags on the context's side stream after the work queued on s so
// far; diags_join makes s wait for it (before anything writes rho, Ex, Ey).
int diags_async(vlp4d_ctx *c, int iter, cudaStream_t s);
int diags_join(vlp4d_ctx *c, cudaStream_t s);
int launch_l2norm(vlp4d_ctx *c, const void *fn, int iter, cudaStream_t s);
// f: the owned planes (slab contexts use the global vy index ivy0 + ivy).
int launch_init_case(vlp4d_ctx *c, void *f, int ic, double amp, double k, double u, cudaStream_t s);
int launch_transpose(const void *in, void *out, int rows, int cols, int elem, cudaStream_t s);
int launch_wait_selftest(vlp4d_ctx *c, long long limit, cudaStream_t s);

}  // namespace vlp4d
