/* vlp4d_b200 — C ABI of the B200 (sm_100a) implementation of the vlp4d
 * semi-Lagrangian hot path from yasahi-hpc/P3-miniapps.
 *
 * Every entry point replaces one function of the reference's single-process
 * CUDA variant (miniapps/vlp4d/thrust); the citation in each comment is the
 * reference interface it stands in for.  The C++ layer in
 * p3-miniapps_b200/cpp/refshim/ re-exports these under the reference's own
 * C++ signatures (Advection::advect_1D_x(Config*, const RealView4D&, ...)).
 *
 * Conventions
 * - The distribution function f is a caller-owned DEVICE buffer of
 *   nx*ny*nvx*nvy elements in the reference's layout_left order: element
 *   (ix, iy, ivx, ivy) sits at ix + nx*(iy + ny*(ivx + nvx*ivy))
 *   (miniapps/vlp4d/thrust/types.hpp:13,33).  Its element type is fixed per
 *   context: VLP4D_F64 (double, as the reference) or VLP4D_F32 (float
 *   storage; displacements, weights' derivation, rho accumulation, the field
 *   solve and diagnostics stay FP64).
 * - 2D fields (rho/phi, Ex, Ey) are FP64 nx*ny device arrays owned by the
 *   context, index ix + nx*iy (miniapps/vlp4d/thrust/efield.hpp:13-16).
 * - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *   stream).  All calls are stream-ordered and asynchronous unless stated;
 *   none allocates device memory after vlp4d_ctx_create except
 *   vlp4d_adjoint_create, which allocates the reverse-mode state.
 * - Every function returns VLP4D_OK (0) or an error code; none exits the
 *   process (the reference's SafeCudaCall exits, lib/Cuda_Helper.hpp:8-16).
 *   vlp4d_last_error() gives a message for the calling thread.
 * - A context is not thread-safe; use one context per host thread/stream.
 */
#ifndef VLP4D_B200_H
#define VLP4D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VLP4D_OK 0
#define VLP4D_ERR_INVALID_ARG 1
#define VLP4D_ERR_CUDA 2
#define VLP4D_ERR_UNSUPPORTED 3
#define VLP4D_ERR_NO_DEVICE 4
#define VLP4D_ERR_IO 5
#define VLP4D_ERR_TIMEOUT 6 /* a kernel's bounded wait for an async copy ran out */
#define VLP4D_ERR_RANGE 7   /* a vlp4d_mpi foot left the interpolation range: the
                               reference's "Time step is too large" exit
                               (miniapps/vlp4d_mpi/thrust/Advection.hpp:21-26) */

#define VLP4D_F64 0
#define VLP4D_F32 1

/* Field selectors for vlp4d_field_ptr. */
#define VLP4D_FIELD_RHO 0 /* rho before field_poisson, phi after it (the
                             reference's irfft2 writes phi into rho_,
                             miniapps/vlp4d/thrust/efield.cpp:102) */
#define VLP4D_FIELD_EX 1
#define VLP4D_FIELD_EY 2

/* Initial conditions for vlp4d_init_case.  2/5/10/20 are the reference's
 * testcases (miniapps/vlp4d/thrust/init.cpp:118-285); 110/120 are the
 * perturbed Maxwellians of the benchmark configurations:
 *   110: (1 + amp cos(k x) + amp cos(k y)) M(vx) M(vy)
 *   120: (1 + amp cos(k x) + amp cos(k y)) 0.5[M(vx-u) + M(vx+u)] M(vy)
 * with M the unit Maxwellian exp(-v^2/2)/sqrt(2 pi). */
#define VLP4D_IC_CYL02 2
#define VLP4D_IC_CYL05 5
#define VLP4D_IC_SLD10 10
#define VLP4D_IC_TSI20 20
#define VLP4D_IC_LANDAU_SUM 110
#define VLP4D_IC_TWO_STREAM 120

/* Mirrors the reference's Domain (miniapps/vlp4d/thrust/config.hpp:8-20);
 * dx is derived as (max - min) / n (init.cpp:77-79). */
typedef struct vlp4d_domain {
  int32_t nxmax[4];   /* nx, ny, nvx, nvy */
  double min_phy[4];
  double max_phy[4];
  double dt;
  int32_t nbiter;     /* number of steps; the diagnostic history holds nbiter+1 entries */
  int32_t ifreq;
  int32_t idcase;     /* field_poisson branch: 2, 6, 10, 20 or other (field.cpp:48-76) */
  int32_t fxvx;
} vlp4d_domain;

typedef struct vlp4d_ctx vlp4d_ctx;

/* Parses a reference input deck (values after each ':' in the fixed order of
 * docs/vlp4d.md:55-86), as import() does (miniapps/vlp4d/thrust/init.cpp:12-82). */
int vlp4d_read_deck(const char *path, vlp4d_domain *out);

/* Allocates the Efield/Diags equivalents on the current CUDA device:
 * replaces `new Efield(conf, {nx, ny})` (efield.cpp:5-37, including the
 * cuFFT plans of lib/Cuda_FFT.hpp:83-159) and `new Diags(conf)`
 * (diags.cpp:6-11). */
int vlp4d_ctx_create(const vlp4d_domain *dom, int dtype, vlp4d_ctx **out);
int vlp4d_ctx_destroy(vlp4d_ctx *ctx);

/* ---- vy-slab decomposition of one run over several processes (one GPU
 * each).  Stands in for the reference's domain decomposition of vlp4d_mpi:
 * Distrib::createDecomposition (miniapps/vlp4d_mpi/thrust/Communication.cpp:10-124),
 * Distrib::exchangeHalo with its pack/unpack (Communication.cpp:471-562)
 * and field_reduce's MPI_Allreduce of rho (miniapps/vlp4d_mpi/thrust/Field.cpp:31-40).
 * Here the run is cut along vy only: a rank owns the global vy planes
 * [ivy0, ivy0 + nvy_local), and an f buffer of its context holds `halo`
 * extra planes on each side, nx*ny*nvx*(nvy_local + 2*halo) elements
 * (vlp4d_f_size), owned planes from plane `halo` on.  Because vy is the
 * slowest index of layout_left, each side's halo is ONE contiguous block
 * that the caller's transport (NCCL send/recv) writes in place: no packing.
 *
 * On a slab context every entry point that takes f reads and writes the
 * owned planes of the buffers given, except the vy sweeps
 * (vlp4d_advect_vy, vlp4d_advect_vxvy), which read the owned AND halo
 * planes of the input (the caller fills the halos from the neighbouring
 * ranks' owned planes first) and write the owned planes of the output.
 * vlp4d_field_rho, vlp4d_advect_xy_moment and vlp4d_advect_xyxy leave in rho
 * the moment of the owned planes only: the caller sums rho over the ranks
 * (an all-reduce of nx*ny doubles) before vlp4d_field_poisson, after which
 * every rank holds the same rho/phi, Ex, Ey and diagnostics.  A vy shift
 * that needs planes beyond the halo sets an error that vlp4d_check
 * reports as VLP4D_ERR_RANGE (nothing outside the buffer is read).
 * vlp4d_step, vlp4d_steps, vlp4d_run, vlp4d_print_fxvx, vlp4d_diags_l2norm,
 * the reverse mode and the vlp4d_mpi entry points return
 * VLP4D_ERR_UNSUPPORTED on slab contexts.
 *
 * dom is the whole run; halo >= 3 (the least any vy shift needs: a shift
 * by d cells reads at most floor(|d|) + 3 planes beyond the owned ones, on
 * the side it comes from) and halo <= nvy_local (halos come from the two
 * neighbouring ranks only). */
int vlp4d_ctx_create_slab(const vlp4d_domain *dom, int dtype, int ivy0, int nvy_local, int halo,
                          vlp4d_ctx **out);
/* Elements of one f buffer of this context (nx*ny*nvx*nvy for an ordinary
 * context, nx*ny*nvx*(nvy_local + 2*halo) for a slab); 0 for NULL. */
size_t vlp4d_f_size(const vlp4d_ctx *ctx);
/* The slab's first owned global plane, owned plane count and halo width
 * (0, nvy, 0 for an ordinary context); any pointer may be NULL. */
int vlp4d_slab_info(const vlp4d_ctx *ctx, int *ivy0, int *nvy_local, int *halo);
const char *vlp4d_last_error(void);
int vlp4d_ctx_dtype(const vlp4d_ctx *ctx);
/* Number of this library's own kernel launches so far in the process
 * (library kernels such as cuFFT's are not counted).  No counterpart in the
 * reference; used to account for launches in benchmarks. */
unsigned long long vlp4d_kernel_launches(void);

/* Device pointer of a context-owned FP64 nx*ny field (VLP4D_FIELD_*). */
int vlp4d_field_ptr(vlp4d_ctx *ctx, int which, double **dev_ptr);

/* Fills f with an initial condition (initcase, init.cpp:118-141). */
int vlp4d_init_case(vlp4d_ctx *ctx, void *f, int ic, double amp, double k, double u, void *stream);

/* Advection::advect_1D_x / _y (miniapps/vlp4d/thrust/advection.hpp:336-360):
 * 1D Lagrange-5 shift along x by dt*vx, along y by dt*vy.  fn and fnp1 must
 * not overlap. */
int vlp4d_advect_x(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream);
int vlp4d_advect_y(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream);
/* Advection::advect_1D_vx / _vy (advection.hpp:362-386): shift along vx by
 * dt*Ex(x,y), along vy by dt*Ey(x,y), reading the context's Ex/Ey. */
int vlp4d_advect_vx(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream);
int vlp4d_advect_vy(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream);

/* Fused pairs of the Strang sequence (timestep.hpp:17-28 and :43-58):
 * advect_1D_x then advect_1D_y in one pass, and advect_1D_vx then
 * advect_1D_vy in one pass.  Equal to the 1D sequence up to FP rounding. */
int vlp4d_advect_xy(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream);
int vlp4d_advect_vxvy(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream);
/* vlp4d_advect_xy followed by field_rho of its result (timestep.hpp:17-31:
 * advect_1D_x, advect_1D_y, field_rho) in one pass: the moment is summed in
 * the pass's epilogue into the context's rho (FP64, fixed summation order),
 * so f is not read a second time. */
int vlp4d_advect_xy_moment(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream);
/* Two x/y shifts by dt in one pass followed by the moment of the result
 * into the context's rho: the last x/y half step of one Strang step and the
 * first of the next (timestep.hpp:50-58 then :17-28 with dt/2 each), the
 * pass vlp4d_steps runs between steps.  The two x shifts are applied as
 * one 11-tap stencil (offset 2m, weights w*w) and likewise the y shifts, y
 * before x (the x and y shifts commute): equal to vlp4d_advect_xy applied
 * twice in exact arithmetic, and to rounding in floating point; rho equals
 * vlp4d_field_rho of the result up to summation order.  Returns VLP4D_ERR_UNSUPPORTED, launching nothing, when the
 * one-pass kernel does not fit the shape or the buffers (nx not a multiple
 * of 4, not 16-byte aligned, shared memory) or VLP4D_KERNELS=generic: the
 * caller then uses two vlp4d_advect_xy calls.  No reference counterpart as a
 * single call. */
int vlp4d_advect_xyxy(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream);

/* field_rho (miniapps/vlp4d/thrust/field.cpp:6-32): rho = dvx*dvy*sum_v f. */
int vlp4d_field_rho(vlp4d_ctx *ctx, const void *fn, void *stream);
/* field_poisson (field.cpp:34-82 -> efield.cpp:43-105): rho -= 1 for cases
 * 10/20, FP64 2D FFT solve; rho then holds phi. */
int vlp4d_field_poisson(vlp4d_ctx *ctx, void *stream);
/* Diags::compute (diags.cpp:13-55) for iteration `iter` (0..nbiter): energy
 * log(sqrt(sum|E|^2 dx dy)) and mass sum(rho)*dx*dy, kept on the device. */
int vlp4d_diags_compute(vlp4d_ctx *ctx, int iter, void *stream);
/* Synchronises the device and reports VLP4D_ERR_TIMEOUT if a fused kernel
 * gave up waiting for one of its asynchronous copies since the last check
 * (the kernel then exits early instead of hanging; its outputs are not
 * valid).  The reference has no counterpart: its launches are unchecked. */
int vlp4d_check(vlp4d_ctx *ctx);

/* Synchronous read of the diagnostic history entries [0, count); includes
 * vlp4d_check. */
int vlp4d_diags_read(vlp4d_ctx *ctx, double *nrj, double *mass, int count);
/* The vlp4d_mpi diagnostics (miniapps/vlp4d_mpi/thrust/Diags.cpp:17-92),
 * kept beside the vlp4d ones.  vlp4d_diags_compute also records, for the
 * same iteration, nrjx = sqrt(0.5 * sum Ex^2 * dx*dy) and
 * nrjy = sqrt(0.5 * sum Ey^2 * dx*dy) (Diags.cpp:63-64; Kahan-compensated
 * FP64 sums).  vlp4d_diags_l2norm records
 * l2norm = sqrt(sum f^2 * dx*dy*dvx*dvy) of the device state fn
 * (Diags::computeL2norm, Diags.cpp:68-92; Kahan-compensated FP64 sums in a
 * fixed order, FP32 or FP64 f, 16-byte aligned).  vlp4d_diags_read_ext
 * synchronises and copies the first `count` values of the three histories
 * (any pointer may be NULL). */
int vlp4d_diags_l2norm(vlp4d_ctx *ctx, const void *fn, int iter, void *stream);
int vlp4d_diags_read_ext(vlp4d_ctx *ctx, double *nrjx, double *nrjy, double *l2norm, int count);

/* Diags::save (diags.cpp:57-68): "t nrj mass" per iteration into `path`. */
int vlp4d_diags_save(vlp4d_ctx *ctx, const char *path);

/* onetimestep (miniapps/vlp4d/thrust/timestep.hpp:14-67) as three fused
 * passes: x/y half step with the rho moment in its epilogue, the field solve
 * and diagnostic `iter`, the vx/vy full step, the x/y half step.  Reads the
 * state from f_state and writes the advanced state into f_next; f_state is
 * used as scratch and holds no meaningful data afterwards, so callers swap
 * the two pointers between steps.  (The reference's six 1D sweeps ping-pong
 * an even number of times and end in fn; three passes end in the other
 * buffer.) */
int vlp4d_step(vlp4d_ctx *ctx, void *f_state, void *f_next, int iter, void *stream);

/* `nsteps` consecutive steps, iterations iter0 .. iter0+nsteps-1 (the time
 * loop of miniapps/vlp4d/thrust/vlp4d.cpp:63-72): the same steps, field
 * solves and diagnostics as nsteps calls of vlp4d_step.  Where
 * vlp4d_steps_joins_xy says so (FP32 contexts, and FP64 contexts whose
 * nx/4 divides 32; VLP4D_XYXY=1/0 at context creation forces it on/off)
 * the last x/y half step of each step and the first of the next
 * (consecutive, with no field solve between them) run as one pass
 * (vlp4d_advect_xyxy's), so the state between steps is never written to
 * memory: 2*nsteps + 1 passes over f instead of 3*nsteps, equal to nsteps
 * vlp4d_step calls to rounding.  With the joining off the result is
 * bit-identical to them.  Reads f_state, writes the final state into
 * f_next; f_state is scratch. */
int vlp4d_steps(vlp4d_ctx *ctx, void *f_state, void *f_next, int iter0, int nsteps, void *stream);
/* 1 when vlp4d_steps joins consecutive x/y half steps on this context (as
 * above), else 0 (also for NULL).  No reference counterpart: lets a caller
 * that runs the stages itself (a vy-slab driver) follow the same schedule. */
int vlp4d_steps_joins_xy(const vlp4d_ctx *ctx);

/* The time loop of main() (miniapps/vlp4d/thrust/vlp4d.cpp:55-73) with host
 * buffers: copies f0 (host, nx*ny*nvx*nvy elements of the context's dtype)
 * into fn, runs the initial field solve + diagnostic 0 and `nsteps` steps,
 * copies the final f back into f_out (host; may be NULL) and the
 * diagnostic history into nrj/mass (host, nsteps+1 entries each; may be
 * NULL).  Synchronous. */
int vlp4d_run(vlp4d_ctx *ctx, const void *f0_host, void *f_out_host, int nsteps, double *nrj,
              double *mass, void *fn, void *fnp1, void *stream);

/* Advection::print_fxvx (advection.hpp:388-411): the (x, vx) slice at iy=0,
 * ivy=nvy/2 as CSV into `path`.  Synchronous. */
int vlp4d_print_fxvx(vlp4d_ctx *ctx, const void *fn, const char *path);

/* field_rho for callers that cannot allocate device memory: callers whose
 * device memory is owned by their own pool allocator, or whose time loop must
 * not pay cudaMalloc/cudaFree (cudaFree synchronises the whole device), and so
 * cannot create a vlp4d_ctx.  No counterpart in the reference.  Computes
 * rho = dvx*dvy*sum_v f (FP64, nx*ny device array) from f (device, dtype
 * VLP4D_F64/VLP4D_F32) without allocating: the reduction's partial sums use a
 * fixed 4 MiB array built into the library (present on every GPU that loads
 * it, until exit), so nx*ny may not exceed 524288 (larger grids return
 * VLP4D_ERR_INVALID_ARG).  The first call on each device, with that device
 * current, looks up the array's device address once and keeps it for the
 * life of the process; make that first call before any stream capture, and
 * do not call this entry point after a cudaDeviceReset of that device (the
 * kept address would be stale).  All calls share the array: calls whose kernels
 * overlap on the GPU race, so issue them on one stream or otherwise in
 * order. */
int vlp4d_field_rho_noalloc(const void *fn, int dtype, int nx, int ny, int nvx, int nvy, double dvx, double dvy,
                            double *rho, void *stream);

/* Impl::Transpose::forward/backward (lib/Cuda_Transpose.hpp:38-46):
 * out-of-place transpose of a (rows x cols) column-major matrix of
 * elements of `elem_size` bytes (4, 8 or 16). */
int vlp4d_transpose(const void *in, void *out, int rows, int cols, int elem_size, void *stream);

/* Self-test of the bounded device waits (no reference counterpart).  The
 * fused kernels wait for their asynchronous copies with a time limit and,
 * when it runs out, record a timeout in the context's error word and
 * return, so a lost copy becomes VLP4D_ERR_TIMEOUT from vlp4d_check instead
 * of a hung GPU.  This launches one thread that waits, with the same
 * primitive, on a barrier phase that nothing completes, for limit_cycles
 * clock cycles (at most the fused kernels' own limit of 4e9); vlp4d_check
 * then returns VLP4D_ERR_TIMEOUT and clears the word; the context stays
 * usable. */
int vlp4d_selftest_wait_timeout(vlp4d_ctx *ctx, long long limit_cycles, void *stream);

/* ---- Reverse mode (discrete adjoint).  No reference counterpart: the
 * reference has no derivative code.  The adjoint is that of vlp4d_step as
 * computed here: transposed interpolation for the x/y shifts, transposed
 * interpolation plus the derivative of the Lagrange weights with respect to
 * E for the vx/vy shifts, back through field_poisson (the transpose of the
 * spectral solve, from its impulse responses) and field_rho.  f, lambda and
 * gradients have the context's element type and layout.
 *
 * The run-level objective is J(f_N) = dx*dy * sum_{x,y} (Ex^2 + Ey^2): the
 * electric energy of the field solved from the state after nsteps steps. */
typedef struct vlp4d_adjoint vlp4d_adjoint;

/* Allocates the reverse-mode state for runs of nsteps steps of ctx with a
 * checkpoint of f every `every` steps: ceil(nsteps/every) checkpoints, every
 * recompute buffers and six work buffers, each one f, plus 2*every fields.
 * The recomputation of a segment therefore holds `every` states at a time.
 * every = 0: no checkpoints; the forward run stores the stage input (one f)
 * and field of each of the nsteps steps, and vlp4d_adjoint_backward
 * recomputes nothing (nsteps + 6 f in all; results bit-identical to
 * every = nsteps).  Runs one field solve on a unit impulse (the context's
 * rho/Ex/Ey are restored). */
int vlp4d_adjoint_create(vlp4d_ctx *ctx, int nsteps, int every, vlp4d_adjoint **out);
int vlp4d_adjoint_destroy(vlp4d_adjoint *adj);

/* nsteps steps from f0 (device, not modified), keeping the checkpoints;
 * the final state is copied to f_out when f_out is not NULL and J receives
 * the objective (host pointer, may be NULL).  Synchronises the stream. */
int vlp4d_adjoint_forward(vlp4d_adjoint *adj, const void *f0, void *f_out, double *J, void *stream);
/* grad = dJ/df0 for the last vlp4d_adjoint_forward; recomputes each segment
 * from its checkpoint (not with every = 0), then runs the reverse steps.
 * Synchronises. */
int vlp4d_adjoint_backward(vlp4d_adjoint *adj, void *grad, void *stream);

/* One reverse step: lam_out = (d step/d f)^T lam_next, the step taken at
 * the state f_state (vlp4d_step's map f_state -> f_next).  lam_out must not
 * alias the inputs.  Overwrites the context's rho/Ex/Ey and v tables. */
int vlp4d_step_adjoint(vlp4d_adjoint *adj, const void *f_state, const void *lam_next, void *lam_out, void *stream);
/* J(f) and lam = dJ/df; J is a host pointer (may be NULL; when given, the
 * call synchronises the stream). */
int vlp4d_energy_grad(vlp4d_adjoint *adj, const void *f, double *J, void *lam, void *stream);

/* ---- Batched ensemble.  No reference counterpart (the reference runs one
 * domain per process).  Many independent runs of uneven grids, each the
 * vlp4d time loop of timestep.hpp:14-67 with FP32 f and FP64 fields (the
 * closing x/y half step of one step and the opening one of the next joined
 * as in vlp4d_steps) from the Landau initial condition
 * f0 = M(vx) M(vy) (1 + amp (cos k x + cos k y)),
 * advance in ONE persistent kernel launch that a CUDA graph replays (with
 * the initial condition and the scheduler reset).  Members need
 * nx, ny, nvx <= 64.  The energy history of each member (nsteps + 1 values,
 * log of the electric-energy norm as Diags::compute) is kept on the device. */
typedef struct {
  int n[4];            /* nx, ny, nvx, nvy */
  double min_phy[4];
  double max_phy[4];
  double dt;
  double amp, k;       /* initial perturbation amplitude and wave number */
} vlp4d_ens_member;
typedef struct vlp4d_ensemble vlp4d_ensemble;

int vlp4d_ensemble_create(const vlp4d_ens_member *members, int nruns, int nsteps, vlp4d_ensemble **out);
int vlp4d_ensemble_destroy(vlp4d_ensemble *ens);
/* Initial condition + nsteps steps of every member (graph replay; the first
 * call captures).  Asynchronous; vlp4d_ensemble_check synchronises and
 * reports VLP4D_ERR_TIMEOUT if a CTA gave up waiting for work. */
int vlp4d_ensemble_run(vlp4d_ensemble *ens, void *stream);
int vlp4d_ensemble_check(vlp4d_ensemble *ens);
/* Final f of member `run` (device copy, FP32, its own layout_left extents)
 * and its energy history (host, nsteps + 1 values); either may be NULL. */
int vlp4d_ensemble_read(vlp4d_ensemble *ens, int run, void *f_out, double *nrj, void *stream);
long long vlp4d_ensemble_cells(const vlp4d_ensemble *ens);
/* Tile configuration: threads per CTA, columns per vx/vy tile, CTAs per SM
 * (0 = as many as fit).  The autotuner scans threads {128, 256, 512},
 * columns {8, 16, 32, 64} and CTAs per SM {1..4}, timing `steps` steps per
 * configuration; it writes one CSV line per configuration to csv_path
 * (NULL: none) and keeps the fastest. */
int vlp4d_ensemble_set_tiles(vlp4d_ensemble *ens, int threads, int cols_per_tile, int ctas_per_sm);
int vlp4d_ensemble_get_tiles(const vlp4d_ensemble *ens, int *threads, int *cols_per_tile, int *ctas_per_sm);
int vlp4d_ensemble_autotune(vlp4d_ensemble *ens, int steps, const char *csv_path, void *stream);
/* How long (clock cycles) a CTA of the persistent kernel looks for a free
 * tile in vain before it flags VLP4D_ERR_TIMEOUT (vlp4d_ensemble_check)
 * and leaves; 0 restores the default and maximum, 4e9 (about two seconds).
 * The CTAs that keep finding work finish the run, so its results stay
 * valid; the flag says that some CTA gave up.  No reference counterpart. */
int vlp4d_ensemble_set_idle_limit(vlp4d_ensemble *ens, long long cycles);

/* ---- vlp4d_mpi, one process (miniapps/vlp4d_mpi, cubic-spline scheme).
 *
 * The arrays are the reference's halo-extended views (RealView4D with
 * offsets, miniapps/vlp4d_mpi/openmp/Init.cpp:333-343): FP64, extents
 * n[d] + 6 in every dimension, first index -3 (HALO_PTS = 3, Config.hpp:7),
 * layout_left, vlp4d_mpi_size() elements, 16-byte aligned.  The context must
 * be FP64 with every grid dimension at least 10 (MMAX + 2, Init.cpp:85-89).
 * A foot outside the interpolation range sets the context's error word:
 * vlp4d_check then returns VLP4D_ERR_RANGE (the reference exits with "Time
 * step is too large", thrust/Advection.hpp:21-26).  All calls are
 * asynchronous on `stream`. */
size_t vlp4d_mpi_size(const vlp4d_ctx *ctx);
/* initcase of vlp4d_mpi (miniapps/vlp4d_mpi/openmp/Init.cpp:126-277) for the
 * domain's idcase: 10 SLD10, 20 TSI20 (vlp4d_mpi's own formula), 2/5 CYL02/
 * CYL05, on the grid points of fn; the halo is zero (Init.cpp:370-372).
 * Another idcase is VLP4D_ERR_INVALID_ARG (the reference aborts). */
int vlp4d_mpi_init_case(vlp4d_ctx *ctx, void *fn, void *stream);
/* Distrib::exchangeHalo for one process (thrust/Communication.cpp, with the
 * spline boundary sums of Communication.hpp boundary_condition): periodic
 * images in the halo, sum_{j=1..8} alpha^j f(...) in its outermost layer.
 * Bit-identical to the reference. */
int vlp4d_mpi_halo_fill(vlp4d_ctx *ctx, void *fn, void *stream);
/* Spline::computeCoeff_xy / computeCoeff_vxvy (thrust/Spline.hpp:61-302):
 * cubic B-spline prefilter along x then y / vx then vy, in place on a
 * halo-filled array.  Bit-identical to the reference. */
int vlp4d_mpi_spline_xy(vlp4d_ctx *ctx, void *fn, void *stream);
int vlp4d_mpi_spline_vxvy(vlp4d_ctx *ctx, void *fn, void *stream);
/* Advection::advect_2D_xy(conf, fn, fn_tmp, dt) (thrust/Advection.hpp:95-226):
 * fn_tmp receives a copy of fn (spline coefficients), fn's grid points the
 * 4x4 spline interpolation at (x - dt vx, y - dt vy).  Bit-identical. */
int vlp4d_mpi_advect_2d(vlp4d_ctx *ctx, void *fn, void *fn_tmp, double dt, void *stream);
/* Advection::advect_4D(conf, ef, fn, tmp_fn, dt) (thrust/Advection.hpp:228-415)
 * with the context's Ex, Ey: tmp_fn receives a copy of fn (4D spline
 * coefficients), fn's grid points the interpolation at the
 * predictor-corrector feet.  Bit-identical. */
int vlp4d_mpi_advect_4d(vlp4d_ctx *ctx, void *fn, void *tmp_fn, double dt, void *stream);
/* field_rho + field_reduce + field_poisson (thrust/Field.cpp) on the grid
 * points of a halo array: the context's rho (then phi), Ex, Ey. */
int vlp4d_mpi_field(vlp4d_ctx *ctx, const void *fn, void *stream);
/* Diags::computeL2norm (thrust/Diags.cpp:68-92) of the grid points of a halo
 * array into history slot iter (read with vlp4d_diags_read_ext). */
int vlp4d_mpi_l2norm(vlp4d_ctx *ctx, const void *fn, int iter, void *stream);
/* onetimestep (thrust/Timestep.hpp:34-97) with dt = the domain's dt: the
 * state in fn's grid points advances into fnp1's grid points; fn is
 * overwritten (it ends holding the 4D spline coefficients, as in the
 * reference) and neither halo is part of the state.  Diagnostic slot `iter`
 * receives the end-of-step nrj, mass, nrjx, nrjy and l2norm (the reference
 * records the mid-step values in the same slot first and then overwrites
 * them).  Fused: four passes over f (x/y prefilter with the 2D advection's
 * moment, vx prefilter, vy prefilter, 4D advection with the moment and the
 * L2 norm); equal to the reference sequence up to FP64 rounding.  The caller
 * swaps fn and fnp1 afterwards, as Vlp4d.cpp:46 does. */
int vlp4d_mpi_step(vlp4d_ctx *ctx, void *fn, void *fnp1, int iter, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* VLP4D_B200_H */
