// The extern "C" entry points of libvlp4d_b200 (include/vlp4d_b200.h).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <atomic>

#include "internal.cuh"
#include "tma.cuh"

namespace vlp4d {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

static std::atomic<unsigned long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

namespace {

int fail(int code, const std::string &msg) {
  set_error(msg);
  return code;
}

bool finite(double v) { return std::isfinite(v); }

// Fallback policy after a fused launcher declined a shape.
int fused_declined(const vlp4d_ctx *c) {
  if (c->fused_only) return fail(VLP4D_ERR_UNSUPPORTED, "fused kernel unavailable for this shape (VLP4D_KERNELS=fused)");
  return VLP4D_OK;
}

int validate_domain(const vlp4d_domain *d) {
  if (!d) return fail(VLP4D_ERR_INVALID_ARG, "domain is NULL");
  long long cells = 1;
  for (int i = 0; i < 4; ++i) {
    if (d->nxmax[i] < 1) return fail(VLP4D_ERR_INVALID_ARG, "nxmax[" + std::to_string(i) + "] < 1");
    if (!finite(d->min_phy[i]) || !finite(d->max_phy[i]) || !(d->max_phy[i] > d->min_phy[i]))
      return fail(VLP4D_ERR_INVALID_ARG, "max_phy[" + std::to_string(i) + "] must exceed min_phy");
    cells *= d->nxmax[i];
    if (cells > (1LL << 40)) return fail(VLP4D_ERR_INVALID_ARG, "grid too large");
  }
  if ((long long)d->nxmax[0] * d->nxmax[1] >= (1LL << 31))
    return fail(VLP4D_ERR_INVALID_ARG, "nx*ny must be below 2^31");
  if (!finite(d->dt)) return fail(VLP4D_ERR_INVALID_ARG, "dt is not finite");
  if (d->nbiter < 0) return fail(VLP4D_ERR_INVALID_ARG, "nbiter < 0");
  return VLP4D_OK;
}

cudaStream_t as_stream(void *s) { return (cudaStream_t)s; }

int check_ctx(const vlp4d_ctx *c) {
  if (!c) return fail(VLP4D_ERR_INVALID_ARG, "context is NULL");
  return VLP4D_OK;
}

int check_pair(const void *a, const void *b) {
  if (!a || !b) return fail(VLP4D_ERR_INVALID_ARG, "f buffer is NULL");
  if (a == b) return fail(VLP4D_ERR_INVALID_ARG, "fn and fnp1 must be different buffers");
  return VLP4D_OK;
}

// Entry points that advance or read a whole run on their own (time loops,
// the reverse mode, the vlp4d_mpi arrays) need every vy plane: slab contexts
// advance through the stage entry points, with the caller's exchanges
// between them.
int reject_slab(const vlp4d_ctx *c, const char *what) {
  if (c->slab)
    return fail(VLP4D_ERR_UNSUPPORTED, std::string(what) + ": not available on a vy-slab context (use the stage "
                                                         "entry points and exchange the halo and rho between ranks)");
  return VLP4D_OK;
}

void free_ctx(vlp4d_ctx *c) {
  if (!c) return;
  if (c->plans) {
    cufftDestroy(c->plan_fwd);
    cufftDestroy(c->plan_bwd);
    cufftDestroy(c->plan_bwd3);
  }
  cudaFree(c->rho);  // ex, ey are slices of this allocation
  cudaFree(c->rho_hat);  // ex_hat, ey_hat likewise
  cudaFree(c->nrj);
  cudaFree(c->nrjx);
  cudaFree(c->l2_part);
  cudaFree(c->mass);
  cudaFree(c->rho_part);
  cudaFree(c->d_err);
  cudaFree(c->mpi_part);
  cudaFree(c->vspan);
  for (StencilTable *t : {&c->tab_x[0], &c->tab_x[1], &c->tab_y[0], &c->tab_y[1], &c->tab_vx, &c->tab_vy,
                          &c->tab_x11, &c->tab_y11}) {
    cudaFree(t->m);
    cudaFree(t->w);
    cudaFree(t->wf);
  }
  if (c->h_diag) cudaFreeHost(c->h_diag);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->side) cudaStreamDestroy(c->side);
  delete c;
}

// Skips to the next ':' as the reference's import() does (init.cpp:35-38),
// returning false at end of file instead of looping forever.
bool skip_to_colon(FILE *f) {
  int ch;
  do {
    ch = fgetc(f);
    if (ch == EOF) return false;
  } while (ch != ':');
  return true;
}

}  // namespace
}  // namespace vlp4d

using namespace vlp4d;

extern "C" {

const char *vlp4d_last_error(void) { return g_last_error.c_str(); }

unsigned long long vlp4d_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

int vlp4d_read_deck(const char *path, vlp4d_domain *out) {
  if (!path || !out) return fail(VLP4D_ERR_INVALID_ARG, "NULL argument");
  FILE *f = fopen(path, "r");
  if (!f) return fail(VLP4D_ERR_IO, std::string("cannot open deck ") + path);
  vlp4d_domain d;
  memset(&d, 0, sizeof(d));
  bool ok = true;
  for (int i = 0; i < 4 && ok; ++i) ok = skip_to_colon(f) && fscanf(f, " %d\n", &d.nxmax[i]) == 1;
  for (int i = 0; i < 4 && ok; ++i) {
    ok = skip_to_colon(f) && fscanf(f, " %le\n", &d.min_phy[i]) == 1;
    ok = ok && skip_to_colon(f) && fscanf(f, " %le\n", &d.max_phy[i]) == 1;
  }
  char idcase[8] = {0};
  ok = ok && skip_to_colon(f) && fgets(idcase, 7, f) != nullptr;
  ok = ok && skip_to_colon(f) && fscanf(f, " %le\n", &d.dt) == 1;
  ok = ok && skip_to_colon(f) && fscanf(f, " %d\n", &d.nbiter) == 1;
  ok = ok && skip_to_colon(f) && fscanf(f, " %d\n", &d.ifreq) == 1;
  ok = ok && skip_to_colon(f) && fscanf(f, " %d\n", &d.fxvx) == 1;
  fclose(f);
  if (!ok) return fail(VLP4D_ERR_IO, std::string("malformed deck ") + path);
  d.idcase = atoi(idcase);
  *out = d;
  return VLP4D_OK;
}

int vlp4d_ctx_create(const vlp4d_domain *dom, int dtype, vlp4d_ctx **out) {
  if (!out) return fail(VLP4D_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  int rc = validate_domain(dom);
  if (rc) return rc;
  if (dtype != VLP4D_F64 && dtype != VLP4D_F32) return fail(VLP4D_ERR_INVALID_ARG, "dtype must be F64 or F32");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return fail(VLP4D_ERR_NO_DEVICE, "no CUDA device");
  }
  vlp4d_ctx *c = new vlp4d_ctx();
  c->dom = *dom;
  c->dtype = dtype;
  c->elem = dtype == VLP4D_F64 ? sizeof(double) : sizeof(float);
  for (int i = 0; i < 4; ++i) {
    c->g.n[i] = dom->nxmax[i];
    c->g.minp[i] = dom->min_phy[i];
    c->g.maxp[i] = dom->max_phy[i];
    c->g.dx[i] = (dom->max_phy[i] - dom->min_phy[i]) / dom->nxmax[i];  // init.cpp:77-79
  }
  c->nvy_glob = c->g.n[3];
  auto bail = [&](int code) {
    free_ctx(c);
    return code;
  };
  if (cudaGetDevice(&c->device) != cudaSuccess) return bail(fail(VLP4D_ERR_CUDA, "cudaGetDevice failed"));
  if (cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess)
    return bail(fail(VLP4D_ERR_CUDA, "cudaDeviceGetAttribute failed"));
  const long long nxy = c->g.nxy();
  const int nx1h = c->g.n[0] / 2 + 1;
  const size_t nh = (size_t)nx1h * c->g.n[1];
#define CTX_ALLOC(ptr, bytes)                                                                \
  do {                                                                                       \
    cudaError_t e_ = cudaMalloc(&(ptr), (bytes));                                            \
    if (e_ != cudaSuccess) return bail(fail(VLP4D_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e_))); \
  } while (0)
  // rho, ex, ey (and their spectra) as 256-byte aligned slices of one
  // allocation, so that one batched inverse transform writes all three.
  c->fstride = (size_t)(nxy + 31) / 32 * 32;
  c->hstride = (nh + 15) / 16 * 16;
  CTX_ALLOC(c->rho, sizeof(double) * 3 * c->fstride);
  c->ex = c->rho + c->fstride;
  c->ey = c->ex + c->fstride;
  CTX_ALLOC(c->rho_hat, sizeof(cufftDoubleComplex) * 3 * c->hstride);
  c->ex_hat = c->rho_hat + c->hstride;
  c->ey_hat = c->ex_hat + c->hstride;
  c->hist_len = dom->nbiter + 1;
  CTX_ALLOC(c->nrj, sizeof(double) * c->hist_len);
  CTX_ALLOC(c->mass, sizeof(double) * c->hist_len);
  CTX_ALLOC(c->nrjx, sizeof(double) * 3 * c->hist_len);
  c->nrjy = c->nrjx + c->hist_len;
  c->l2norm = c->nrjy + c->hist_len;
  c->l2_blocks = 2 * c->num_sms;
  CTX_ALLOC(c->l2_part, sizeof(double) * 2 * c->l2_blocks);
  // Enough (column block, plane group) blocks to fill the GPU a few times.
  long long groups = ((long long)c->num_sms * 8 * 256 + nxy - 1) / nxy;
  if (groups > c->g.nv()) groups = c->g.nv();
  if (groups > 1024) groups = 1024;
  if (groups < 1) groups = 1;
  c->rho_groups = (int)groups;
  // The fused x/y pass writes one partial per plane group (up to two CTAs
  // per SM); bounded so the partials stay below 256 MB.
  long long fused_groups = 2LL * c->num_sms;
  const long long cap = (256LL << 20) / ((long long)sizeof(double) * nxy);
  if (fused_groups > cap) fused_groups = cap;
  c->rho_part_groups = (int)(fused_groups > groups ? fused_groups : groups);
  CTX_ALLOC(c->rho_part, sizeof(double) * nxy * (size_t)c->rho_part_groups);
  CTX_ALLOC(c->d_err, sizeof(int));
  c->mpi_part_cap = 8192;
  CTX_ALLOC(c->mpi_part, sizeof(double) * 2 * (size_t)c->mpi_part_cap);
  c->vspan_cap = (int)(nxy / 8 + 1);
  CTX_ALLOC(c->vspan, sizeof(int2) * (size_t)c->vspan_cap);
  {
    const char *k = getenv("VLP4D_KERNELS");
    c->fused = !(k && strcmp(k, "generic") == 0);
    c->fused_only = k && strcmp(k, "fused") == 0;
    const char *xx = getenv("VLP4D_XYXY");
    if (xx && *xx) c->xyxy_mode = atoi(xx) ? 1 : 0;
  }
#undef CTX_ALLOC
  if (cudaMemset(c->rho, 0, sizeof(double) * nxy) != cudaSuccess ||
      cudaMemset(c->ex, 0, sizeof(double) * nxy) != cudaSuccess ||
      cudaMemset(c->ey, 0, sizeof(double) * nxy) != cudaSuccess ||
      cudaMemset(c->nrj, 0, sizeof(double) * c->hist_len) != cudaSuccess ||
      cudaMemset(c->mass, 0, sizeof(double) * c->hist_len) != cudaSuccess ||
      cudaMemset(c->nrjx, 0, sizeof(double) * 3 * c->hist_len) != cudaSuccess ||
      cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess)
    return bail(fail(VLP4D_ERR_CUDA, "cudaMemset failed"));
  // lib/Cuda_FFT.hpp:108-114: cufftPlan2d(nx2 = ny, nx1 = nx) on x-fastest data.
  if (cufftPlan2d(&c->plan_fwd, c->g.n[1], c->g.n[0], CUFFT_D2Z) != CUFFT_SUCCESS)
    return bail(fail(VLP4D_ERR_CUDA, "cufftPlan2d D2Z failed"));
  if (cufftPlan2d(&c->plan_bwd, c->g.n[1], c->g.n[0], CUFFT_Z2D) != CUFFT_SUCCESS) {
    cufftDestroy(c->plan_fwd);
    return bail(fail(VLP4D_ERR_CUDA, "cufftPlan2d Z2D failed"));
  }
  {
    int n[2] = {c->g.n[1], c->g.n[0]};
    int inembed[2] = {c->g.n[1], nx1h}, onembed[2] = {c->g.n[1], c->g.n[0]};
    if (cufftPlanMany(&c->plan_bwd3, 2, n, inembed, 1, (int)c->hstride, onembed, 1, (int)c->fstride, CUFFT_Z2D, 3) !=
        CUFFT_SUCCESS) {
      cufftDestroy(c->plan_fwd);
      cufftDestroy(c->plan_bwd);
      return bail(fail(VLP4D_ERR_CUDA, "cufftPlanMany Z2D (batch 3) failed"));
    }
  }
  c->plans = true;
  if (cudaMallocHost(&c->h_diag, sizeof(double) * 2 * c->hist_len) != cudaSuccess)
    return bail(fail(VLP4D_ERR_CUDA, "cudaMallocHost failed"));
  if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(VLP4D_ERR_CUDA, "stream/event creation failed"));
  *out = c;
  return VLP4D_OK;
}

int vlp4d_ctx_create_slab(const vlp4d_domain *dom, int dtype, int ivy0, int nvy_local, int halo, vlp4d_ctx **out) {
  if (!out) return fail(VLP4D_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  int rc = validate_domain(dom);
  if (rc) return rc;
  const int nvy = dom->nxmax[3];
  if (nvy_local < 1 || ivy0 < 0 || (long long)ivy0 + nvy_local > nvy)
    return fail(VLP4D_ERR_INVALID_ARG, "slab planes [ivy0, ivy0 + nvy_local) must lie in [0, nvy)");
  // Three halo planes are the least any vy shift needs: a shift by d cells,
  // |d| < 1, reads the six planes from ivy-3 (d > 0) or ivy-2 (d <= 0) on.
  // In general a shift by d reads at most floor(|d|) + 3 planes beyond the
  // owned ones, on the side it comes from.
  if (halo < 3) return fail(VLP4D_ERR_INVALID_ARG, "halo must be at least 3 planes");
  if (halo > nvy_local) return fail(VLP4D_ERR_INVALID_ARG, "halo wider than the slab (neighbours' planes only)");
  if (halo > nvy) return fail(VLP4D_ERR_INVALID_ARG, "halo wider than the run");
  vlp4d_domain local = *dom;
  local.nxmax[3] = nvy_local;
  long long ext = (long long)dom->nxmax[0] * dom->nxmax[1] * dom->nxmax[2] * (nvy_local + 2LL * halo);
  if (ext > (1LL << 40)) return fail(VLP4D_ERR_INVALID_ARG, "grid too large");
  vlp4d_ctx *c = nullptr;
  if ((rc = vlp4d_ctx_create(&local, dtype, &c))) return rc;
  c->dom = *dom;
  c->slab = true;
  c->ivy0 = ivy0;
  c->halo = halo;
  c->nvy_glob = nvy;
  // The vy geometry of the whole run: coordinates and tables of the owned
  // planes use their global index.
  c->g.minp[3] = dom->min_phy[3];
  c->g.maxp[3] = dom->max_phy[3];
  c->g.dx[3] = (dom->max_phy[3] - dom->min_phy[3]) / nvy;
  *out = c;
  return VLP4D_OK;
}

size_t vlp4d_f_size(const vlp4d_ctx *ctx) {
  if (!ctx) return 0;
  return vy_plane_elems(ctx) * (size_t)(ctx->g.n[3] + 2 * ctx->halo);
}

int vlp4d_slab_info(const vlp4d_ctx *ctx, int *ivy0, int *nvy_local, int *halo) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (ivy0) *ivy0 = ctx->ivy0;
  if (nvy_local) *nvy_local = ctx->g.n[3];
  if (halo) *halo = ctx->halo;
  return VLP4D_OK;
}

int vlp4d_ctx_destroy(vlp4d_ctx *ctx) {
  if (!ctx) return VLP4D_OK;
  free_ctx(ctx);
  return VLP4D_OK;
}

int vlp4d_ctx_dtype(const vlp4d_ctx *ctx) { return ctx ? ctx->dtype : -1; }

int vlp4d_steps_joins_xy(const vlp4d_ctx *ctx) { return ctx && xyxy_join(ctx) ? 1 : 0; }

int vlp4d_field_ptr(vlp4d_ctx *ctx, int which, double **dev_ptr) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!dev_ptr) return fail(VLP4D_ERR_INVALID_ARG, "dev_ptr is NULL");
  switch (which) {
    case VLP4D_FIELD_RHO: *dev_ptr = ctx->rho; break;
    case VLP4D_FIELD_EX: *dev_ptr = ctx->ex; break;
    case VLP4D_FIELD_EY: *dev_ptr = ctx->ey; break;
    default: return fail(VLP4D_ERR_INVALID_ARG, "unknown field");
  }
  return VLP4D_OK;
}

int vlp4d_init_case(vlp4d_ctx *ctx, void *f, int ic, double amp, double k, double u, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!f) return fail(VLP4D_ERR_INVALID_ARG, "f is NULL");
  switch (ic) {
    case VLP4D_IC_CYL02: case VLP4D_IC_CYL05: case VLP4D_IC_SLD10: case VLP4D_IC_TSI20:
    case VLP4D_IC_LANDAU_SUM: case VLP4D_IC_TWO_STREAM: break;
    default: return fail(VLP4D_ERR_INVALID_ARG, "unknown initial condition");  // init.cpp:135-138 aborts
  }
  return launch_init_case(ctx, owned_planes(ctx, f), ic, amp, k, u, as_stream(stream));
}

static int advect_vxvy_impl(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, cudaStream_t s);

// The vy sweep (after the vx sweep when do_vx) of a slab context: reads the
// whole input buffer fn_ext (owned planes and filled halos), writes the
// owned planes of fnp1_owned.
static int slab_vy(vlp4d_ctx *ctx, const void *fn_ext, void *fnp1_owned, bool do_vx, cudaStream_t s) {
  int rc = launch_advect_vxvy_tables(ctx, fn_ext, fnp1_owned, do_vx ? &ctx->tab_vx : nullptr, &ctx->tab_vy, s);
  if (rc != VLP4D_ERR_UNSUPPORTED) return rc;
  if ((rc = fused_declined(ctx))) return rc;
  return launch_vy_slab_generic(ctx, fn_ext, fnp1_owned, do_vx ? &ctx->tab_vx : nullptr, &ctx->tab_vy, s);
}

static int advect_1d(vlp4d_ctx *ctx, int dim, const void *fn_buf, void *fnp1_buf, double dt, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = check_pair(fn_buf, fnp1_buf))) return rc;
  if (!std::isfinite(dt)) return fail(VLP4D_ERR_INVALID_ARG, "dt is not finite");
  cudaStream_t s = as_stream(stream);
  // Owned planes of slab buffers (the buffers themselves otherwise).
  const void *fn = owned_planes(ctx, fn_buf);
  void *fnp1 = owned_planes(ctx, fnp1_buf);
  StencilTable *t = nullptr;
  if (dim < 2) {
    if ((rc = ensure_xy_table(ctx, dim, dt, &t, s))) return rc;
    rc = launch_advect_xy(ctx, fn, fnp1, dim == 0 ? t : nullptr, dim == 1 ? t : nullptr, dim == 0, dim == 1,
                          false, s);
    if (rc != VLP4D_ERR_UNSUPPORTED) return rc;
    if ((rc = fused_declined(ctx))) return rc;
    return launch_advect_generic(ctx, dim, fn, fnp1, t, s);
  }
  if ((rc = build_v_tables(ctx, dt, dim == 2, dim == 3, s))) return rc;
  if (dim == 3 && ctx->slab) return slab_vy(ctx, fn_buf, fnp1, false, s);
  rc = launch_advect_vxvy(ctx, fn, fnp1, dim == 2, dim == 3, s);
  if (rc != VLP4D_ERR_UNSUPPORTED) return rc;
  if ((rc = fused_declined(ctx))) return rc;
  return launch_advect_generic(ctx, dim, fn, fnp1, dim == 2 ? &ctx->tab_vx : &ctx->tab_vy, s);
}

int vlp4d_advect_x(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream) {
  return advect_1d(ctx, 0, fn, fnp1, dt, stream);
}
int vlp4d_advect_y(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream) {
  return advect_1d(ctx, 1, fn, fnp1, dt, stream);
}
int vlp4d_advect_vx(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream) {
  return advect_1d(ctx, 2, fn, fnp1, dt, stream);
}
int vlp4d_advect_vy(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream) {
  return advect_1d(ctx, 3, fn, fnp1, dt, stream);
}

static int advect_xy_impl(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, bool with_rho, cudaStream_t s) {
  StencilTable *tx = nullptr, *ty = nullptr;
  int rc;
  if ((rc = ensure_xy_table(ctx, 0, dt, &tx, s))) return rc;
  if ((rc = ensure_xy_table(ctx, 1, dt, &ty, s))) return rc;
  rc = launch_advect_xy(ctx, fn, fnp1, tx, ty, true, true, with_rho, s);
  if (rc != VLP4D_ERR_UNSUPPORTED) return rc;
  if ((rc = fused_declined(ctx))) return rc;
  if ((rc = launch_advect_pair_generic(ctx, false, fn, fnp1, tx, ty, s))) return rc;
  return with_rho ? launch_field_rho(ctx, fnp1, s) : VLP4D_OK;
}

// Slab contexts: fn is the whole input buffer, fnp1 the owned output planes.
static int advect_vxvy_impl(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, cudaStream_t s) {
  int rc;
  if ((rc = build_v_tables(ctx, dt, true, true, s))) return rc;
  if (ctx->slab) return slab_vy(ctx, fn, fnp1, true, s);
  rc = launch_advect_vxvy(ctx, fn, fnp1, true, true, s);
  if (rc != VLP4D_ERR_UNSUPPORTED) return rc;
  if ((rc = fused_declined(ctx))) return rc;
  return launch_advect_pair_generic(ctx, true, fn, fnp1, &ctx->tab_vx, &ctx->tab_vy, s);
}

int vlp4d_advect_xy(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = check_pair(fn, fnp1))) return rc;
  if (!std::isfinite(dt)) return fail(VLP4D_ERR_INVALID_ARG, "dt is not finite");
  return advect_xy_impl(ctx, owned_planes(ctx, fn), owned_planes(ctx, fnp1), dt, false, as_stream(stream));
}

int vlp4d_advect_xy_moment(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = check_pair(fn, fnp1))) return rc;
  if (!std::isfinite(dt)) return fail(VLP4D_ERR_INVALID_ARG, "dt is not finite");
  return advect_xy_impl(ctx, owned_planes(ctx, fn), owned_planes(ctx, fnp1), dt, true, as_stream(stream));
}

int vlp4d_advect_xyxy(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = check_pair(fn, fnp1))) return rc;
  if (!std::isfinite(dt)) return fail(VLP4D_ERR_INVALID_ARG, "dt is not finite");
  cudaStream_t s = as_stream(stream);
  StencilTable *tx = nullptr, *ty = nullptr;
  if ((rc = ensure_xy_table(ctx, 0, dt, &tx, s))) return rc;
  if ((rc = ensure_xy_table(ctx, 1, dt, &ty, s))) return rc;
  rc = launch_advect_xyxy(ctx, owned_planes(ctx, fn), owned_planes(ctx, fnp1), tx, ty, s);
  if (rc == VLP4D_ERR_UNSUPPORTED)
    return fail(rc, "advect_xyxy: the one-pass kernel does not fit this shape, these buffers or VLP4D_KERNELS; "
                    "call vlp4d_advect_xy twice");
  return rc;
}

int vlp4d_advect_vxvy(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = check_pair(fn, fnp1))) return rc;
  if (!std::isfinite(dt)) return fail(VLP4D_ERR_INVALID_ARG, "dt is not finite");
  // Slab contexts: the whole input buffer (halos filled), the owned output planes.
  return advect_vxvy_impl(ctx, fn, owned_planes(ctx, fnp1), dt, as_stream(stream));
}

int vlp4d_field_rho(vlp4d_ctx *ctx, const void *fn, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!fn) return fail(VLP4D_ERR_INVALID_ARG, "fn is NULL");
  return launch_field_rho(ctx, owned_planes(ctx, fn), as_stream(stream));
}

int vlp4d_field_poisson(vlp4d_ctx *ctx, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  return launch_field_poisson(ctx, as_stream(stream));
}

int vlp4d_diags_compute(vlp4d_ctx *ctx, int iter, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  // diags.cpp:17 asserts 0 <= iter <= nbiter.
  if (iter < 0 || iter >= ctx->hist_len) return fail(VLP4D_ERR_INVALID_ARG, "iter outside [0, nbiter]");
  return launch_diags(ctx, iter, as_stream(stream));
}

int vlp4d_check(vlp4d_ctx *ctx) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  VLP4D_CUDA_TRY(cudaDeviceSynchronize());
  int flag = 0;
  VLP4D_CUDA_TRY(cudaMemcpy(&flag, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) {
    VLP4D_CUDA_TRY(cudaMemset(ctx->d_err, 0, sizeof(int)));
    if (flag & kErrTimeout) return fail(VLP4D_ERR_TIMEOUT, "an asynchronous copy did not complete within its time limit");
    if (flag & kErrSlabHalo)
      return fail(VLP4D_ERR_RANGE, "a vy shift needed planes beyond the slab's halo (create the slab with a wider halo)");
    return fail(VLP4D_ERR_RANGE, "a foot left the interpolation range (the reference stops: time step is too large)");
  }
  return VLP4D_OK;
}

int vlp4d_diags_read(vlp4d_ctx *ctx, double *nrj, double *mass, int count) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (count < 0 || count > ctx->hist_len) return fail(VLP4D_ERR_INVALID_ARG, "count outside [0, nbiter+1]");
  if ((rc = vlp4d_check(ctx))) return rc;
  if (nrj) VLP4D_CUDA_TRY(cudaMemcpy(nrj, ctx->nrj, sizeof(double) * count, cudaMemcpyDeviceToHost));
  if (mass) VLP4D_CUDA_TRY(cudaMemcpy(mass, ctx->mass, sizeof(double) * count, cudaMemcpyDeviceToHost));
  return VLP4D_OK;
}

int vlp4d_diags_l2norm(vlp4d_ctx *ctx, const void *fn, int iter, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!fn) return fail(VLP4D_ERR_INVALID_ARG, "fn is NULL");
  if (iter < 0 || iter >= ctx->hist_len) return fail(VLP4D_ERR_INVALID_ARG, "iter outside [0, nbiter]");
  if ((rc = reject_slab(ctx, "diags_l2norm"))) return rc;
  return launch_l2norm(ctx, fn, iter, as_stream(stream));
}

int vlp4d_diags_read_ext(vlp4d_ctx *ctx, double *nrjx, double *nrjy, double *l2norm, int count) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (count < 0 || count > ctx->hist_len) return fail(VLP4D_ERR_INVALID_ARG, "count outside [0, nbiter+1]");
  if ((rc = vlp4d_check(ctx))) return rc;
  if (nrjx) VLP4D_CUDA_TRY(cudaMemcpy(nrjx, ctx->nrjx, sizeof(double) * count, cudaMemcpyDeviceToHost));
  if (nrjy) VLP4D_CUDA_TRY(cudaMemcpy(nrjy, ctx->nrjy, sizeof(double) * count, cudaMemcpyDeviceToHost));
  if (l2norm) VLP4D_CUDA_TRY(cudaMemcpy(l2norm, ctx->l2norm, sizeof(double) * count, cudaMemcpyDeviceToHost));
  return VLP4D_OK;
}

int vlp4d_diags_save(vlp4d_ctx *ctx, const char *path) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!path) return fail(VLP4D_ERR_INVALID_ARG, "path is NULL");
  const int n = ctx->hist_len;
  double *buf = (double *)malloc(sizeof(double) * 2 * n);
  if ((rc = vlp4d_diags_read(ctx, buf, buf + n, n))) {
    free(buf);
    return rc;
  }
  FILE *f = fopen(path, "w");
  if (!f) {
    free(buf);
    return fail(VLP4D_ERR_IO, std::string("cannot write ") + path);
  }
  for (int it = 0; it < n; ++it)  // diags.cpp:64-65
    fprintf(f, "%17.13e %17.13e %17.13e\n", it * ctx->dom.dt, buf[it], buf[n + it]);
  fclose(f);
  free(buf);
  return VLP4D_OK;
}

}  // extern "C"

namespace vlp4d {

// One Strang step f_in -> f_out through `scratch` (f_in is left unchanged
// when scratch != f_in); the mid-step diagnostic goes to history slot
// `iter`, or nowhere when iter < 0.
int step_impl(vlp4d_ctx *ctx, const void *f_in, void *f_out, void *scratch, int iter, cudaStream_t s) {
  const double dt = ctx->dom.dt;
  int rc;
  // timestep.hpp:17-28: x(dt/2), y(dt/2) and the moment of the result.
  if ((rc = advect_xy_impl(ctx, f_in, f_out, 0.5 * dt, true, s))) return rc;
  // timestep.hpp:30-38: field solve and the mid-step diagnostic (beside
  // the v pass, on the side stream).
  if ((rc = launch_field_poisson(ctx, s))) return rc;
  if (iter >= 0 && (rc = diags_async(ctx, iter, s))) return rc;
  // timestep.hpp:40-48: vx(dt), vy(dt).
  if ((rc = advect_vxvy_impl(ctx, f_out, scratch, dt, s))) return rc;
  // timestep.hpp:50-58: x(dt/2), y(dt/2).
  if ((rc = advect_xy_impl(ctx, scratch, f_out, 0.5 * dt, false, s))) return rc;
  return iter >= 0 ? diags_join(ctx, s) : VLP4D_OK;
}

int advect_xy_moment(vlp4d_ctx *ctx, const void *fn, void *fnp1, double dt, cudaStream_t s) {
  return advect_xy_impl(ctx, fn, fnp1, dt, true, s);
}

int advect_xy_any(vlp4d_ctx *ctx, const void *fn, void *fnp1, const StencilTable *tx, const StencilTable *ty,
                  cudaStream_t s) {
  int rc = launch_advect_xy(ctx, fn, fnp1, tx, ty, true, true, false, s);
  if (rc != VLP4D_ERR_UNSUPPORTED) return rc;
  if ((rc = fused_declined(ctx))) return rc;
  return launch_advect_pair_generic(ctx, false, fn, fnp1, tx, ty, s);
}

int advect_vxvy_any(vlp4d_ctx *ctx, const void *fn, void *fnp1, const StencilTable *tvx, const StencilTable *tvy,
                    cudaStream_t s) {
  int rc = launch_advect_vxvy_tables(ctx, fn, fnp1, tvx, tvy, s);
  if (rc != VLP4D_ERR_UNSUPPORTED) return rc;
  if ((rc = fused_declined(ctx))) return rc;
  return launch_advect_pair_generic(ctx, true, fn, fnp1, tvx, tvy, s);
}

int fail_msg(int code, const std::string &msg) { return fail(code, msg); }

// Whether the x/y half steps of consecutive steps run as one joined pass.
// That pass does the arithmetic of two passes for the HBM traffic of one:
// in FP32 (k_plane_xyxy, 0.50 ms against 2 x 0.41 ms at 128^4) and in FP64
// where k_plane_xyxy64 runs (1.08 ms against 2 x 0.84 ms), not for the FP64
// widths only the generic FP64 form covers (its 1 KB rows leave one CTA per
// SM: slower than two k_plane passes).  VLP4D_XYXY=0/1 at context creation
// overrides.
bool xyxy_join(const vlp4d_ctx *ctx) {
  if (ctx->xyxy_mode >= 0) return ctx->xyxy_mode == 1;
  return ctx->dtype == VLP4D_F32 || xyxy64_available(ctx);
}

}  // namespace vlp4d

extern "C" {

int vlp4d_step(vlp4d_ctx *ctx, void *f_state, void *f_next, int iter, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = check_pair(f_state, f_next))) return rc;
  if (iter < 0 || iter >= ctx->hist_len) return fail(VLP4D_ERR_INVALID_ARG, "iter outside [0, nbiter]");
  if ((rc = reject_slab(ctx, "step"))) return rc;
  return step_impl(ctx, f_state, f_next, f_state, iter, as_stream(stream));
}

// The reference's time loop (vlp4d.cpp:63-72, onetimestep per step) with
// the last x/y half step of each step fused with the first of the next.
int vlp4d_steps(vlp4d_ctx *ctx, void *f_state, void *f_next, int iter0, int nsteps, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = check_pair(f_state, f_next))) return rc;
  if (nsteps < 1) return fail(VLP4D_ERR_INVALID_ARG, "nsteps must be at least 1");
  if (iter0 < 0 || (long long)iter0 + nsteps - 1 >= ctx->hist_len)
    return fail(VLP4D_ERR_INVALID_ARG, "iterations outside [0, nbiter]");
  if ((rc = reject_slab(ctx, "steps"))) return rc;
  cudaStream_t s = as_stream(stream);
  const double dt = ctx->dom.dt;
  StencilTable *tx = nullptr, *ty = nullptr;
  if ((rc = ensure_xy_table(ctx, 0, 0.5 * dt, &tx, s))) return rc;
  if ((rc = ensure_xy_table(ctx, 1, 0.5 * dt, &ty, s))) return rc;
  void *cur = f_state, *oth = f_next;
  // timestep.hpp:17-28 of the first step: x/y half step and the moment.
  if ((rc = advect_xy_impl(ctx, cur, oth, 0.5 * dt, true, s))) return rc;
  std::swap(cur, oth);
  for (int k = 0; k < nsteps; ++k) {
    // timestep.hpp:30-48: field solve, diagnostic (on the side stream,
    // beside the v pass), vx/vy full step.
    if ((rc = launch_field_poisson(ctx, s))) return rc;
    if ((rc = diags_async(ctx, iter0 + k, s))) return rc;
    if ((rc = advect_vxvy_impl(ctx, cur, oth, dt, s))) return rc;
    std::swap(cur, oth);
    // The diagnostic has read rho and the field before the next pass
    // writes rho (or before the call returns).
    if ((rc = diags_join(ctx, s))) return rc;
    if (k + 1 == nsteps) break;
    // timestep.hpp:50-58 of step k, then :17-28 of step k+1, in one pass
    // where that pass is the faster choice.
    rc = xyxy_join(ctx) ? launch_advect_xyxy(ctx, cur, oth, tx, ty, s) : VLP4D_ERR_UNSUPPORTED;
    if (rc == VLP4D_ERR_UNSUPPORTED && !xyxy_join(ctx)) {
      if ((rc = advect_xy_impl(ctx, cur, oth, 0.5 * dt, false, s))) return rc;
      std::swap(cur, oth);
      if ((rc = advect_xy_impl(ctx, cur, oth, 0.5 * dt, true, s))) return rc;
    } else if (rc == VLP4D_ERR_UNSUPPORTED) {
      if ((rc = fused_declined(ctx))) return rc;
      if ((rc = advect_xy_impl(ctx, cur, oth, 0.5 * dt, false, s))) return rc;
      std::swap(cur, oth);
      if ((rc = advect_xy_impl(ctx, cur, oth, 0.5 * dt, true, s))) return rc;
    } else if (rc) {
      return rc;
    }
    std::swap(cur, oth);
  }
  // timestep.hpp:50-58 of the last step.
  if ((rc = advect_xy_impl(ctx, cur, oth, 0.5 * dt, false, s))) return rc;
  std::swap(cur, oth);
  if (cur != f_next)
    VLP4D_CUDA_TRY(cudaMemcpyAsync(f_next, cur, (size_t)ctx->g.cells() * ctx->elem, cudaMemcpyDeviceToDevice, s));
  return VLP4D_OK;
}

int vlp4d_run(vlp4d_ctx *ctx, const void *f0_host, void *f_out_host, int nsteps, double *nrj, double *mass,
              void *fn, void *fnp1, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if ((rc = check_pair(fn, fnp1))) return rc;
  if (!f0_host) return fail(VLP4D_ERR_INVALID_ARG, "f0_host is NULL");
  if (nsteps < 0 || nsteps >= ctx->hist_len) return fail(VLP4D_ERR_INVALID_ARG, "nsteps outside [0, nbiter]");
  if ((rc = reject_slab(ctx, "run"))) return rc;
  cudaStream_t s = as_stream(stream);
  const size_t bytes = (size_t)ctx->g.cells() * ctx->elem;
  VLP4D_CUDA_TRY(cudaMemcpyAsync(fn, f0_host, bytes, cudaMemcpyHostToDevice, s));
  // vlp4d.cpp:58-61: initial moment, field and diagnostic 0.
  if ((rc = launch_field_rho(ctx, fn, s))) return rc;
  if ((rc = launch_field_poisson(ctx, s))) return rc;
  if ((rc = launch_diags(ctx, 0, s))) return rc;
  void *cur = fn;
  if (nsteps > 0) {
    if ((rc = vlp4d_steps(ctx, fn, fnp1, 1, nsteps, stream))) return rc;
    cur = fnp1;
  }
  if (nrj || mass) {
    VLP4D_CUDA_TRY(cudaMemcpyAsync(ctx->h_diag, ctx->nrj, sizeof(double) * (nsteps + 1), cudaMemcpyDeviceToHost, s));
    VLP4D_CUDA_TRY(cudaMemcpyAsync(ctx->h_diag + ctx->hist_len, ctx->mass, sizeof(double) * (nsteps + 1),
                                   cudaMemcpyDeviceToHost, s));
  }
  if (f_out_host) VLP4D_CUDA_TRY(cudaMemcpyAsync(f_out_host, cur, bytes, cudaMemcpyDeviceToHost, s));
  VLP4D_CUDA_TRY(cudaStreamSynchronize(s));
  if ((rc = vlp4d_check(ctx))) return rc;
  if (nrj) memcpy(nrj, ctx->h_diag, sizeof(double) * (nsteps + 1));
  if (mass) memcpy(mass, ctx->h_diag + ctx->hist_len, sizeof(double) * (nsteps + 1));
  // Leave the final state in fn, as the reference's loop does.
  if (cur != fn) VLP4D_CUDA_TRY(cudaMemcpyAsync(fn, cur, bytes, cudaMemcpyDeviceToDevice, s));
  VLP4D_CUDA_TRY(cudaStreamSynchronize(s));
  return VLP4D_OK;
}

int vlp4d_print_fxvx(vlp4d_ctx *ctx, const void *fn, const char *path) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!fn || !path) return fail(VLP4D_ERR_INVALID_ARG, "NULL argument");
  if ((rc = reject_slab(ctx, "print_fxvx"))) return rc;
  const int nx = ctx->g.n[0], nvx = ctx->g.n[2];
  const int ivy = ctx->g.n[3] / 2;  // advection.hpp:394-395
  const size_t e = ctx->elem;
  const size_t row_pitch = (size_t)ctx->g.nxy() * e;  // consecutive ivx at iy = 0
  const char *base = (const char *)fn + (size_t)ivy * nvx * row_pitch;
  char *h = (char *)malloc((size_t)nx * nvx * e);
  cudaError_t err = cudaMemcpy2D(h, (size_t)nx * e, base, row_pitch, (size_t)nx * e, nvx, cudaMemcpyDeviceToHost);
  if (err != cudaSuccess) {
    free(h);
    return fail(VLP4D_ERR_CUDA, std::string("cudaMemcpy2D: ") + cudaGetErrorString(err));
  }
  FILE *f = fopen(path, "w");
  if (!f) {
    free(h);
    return fail(VLP4D_ERR_IO, std::string("cannot write ") + path);
  }
  for (int ivx = 0; ivx < nvx; ++ivx)
    for (int ix = 0; ix < nx; ++ix) {
      const size_t i = (size_t)ivx * nx + ix;
      const double v = ctx->dtype == VLP4D_F64 ? ((const double *)h)[i] : (double)((const float *)h)[i];
      fprintf(f, ix == nx - 1 ? "%20.13le\n" : "%20.13le, ", v);
    }
  fclose(f);
  free(h);
  return VLP4D_OK;
}

int vlp4d_selftest_wait_timeout(vlp4d_ctx *ctx, long long limit_cycles, void *stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (limit_cycles < 0 || limit_cycles > kWaitCycles)
    return fail(VLP4D_ERR_INVALID_ARG, "limit_cycles outside [0, the fused kernels' own limit]");
  return launch_wait_selftest(ctx, limit_cycles, as_stream(stream));
}

int vlp4d_transpose(const void *in, void *out, int rows, int cols, int elem_size, void *stream) {
  if (!in || !out) return fail(VLP4D_ERR_INVALID_ARG, "NULL buffer");
  if (rows < 1 || cols < 1) return fail(VLP4D_ERR_INVALID_ARG, "rows and cols must be positive");
  if (elem_size != 4 && elem_size != 8 && elem_size != 16)
    return fail(VLP4D_ERR_INVALID_ARG, "elem_size must be 4, 8 or 16");
  if (in == out) return fail(VLP4D_ERR_INVALID_ARG, "transpose is out of place");
  return launch_transpose(in, out, rows, cols, elem_size, as_stream(stream));
}

}  // extern "C"
