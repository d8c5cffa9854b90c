// Velocity moment, FP64 field solve, diagnostics, initial conditions and the
// 2D transpose of the vlp4d hot path.
//
// References: field_rho (miniapps/vlp4d/thrust/field.cpp:6-32),
// field_poisson (field.cpp:34-82) -> Efield::solve_poisson_fftw
// (efield.cpp:43-105) on cuFFT plans (lib/Cuda_FFT.hpp:83-183),
// Diags::compute (diags.cpp:13-55), initcase (init.cpp:118-285),
// Impl::Transpose (lib/Cuda_Transpose.hpp:18-136).
#include "internal.cuh"
#include "moment.cuh"
#include "poisson.cuh"
#include "tma.cuh"

namespace vlp4d {

namespace {

// ---- field_rho: deterministic two-level sum over the (vx, vy) planes.
// Stage 1: block (chunk of columns, group of planes) -> partial[group][ixy].
// Stage 2: rho[ixy] = (sum over groups) * dvx * dvy.
template <typename T>
__global__ void k_rho_partial(const T *__restrict__ f, double *__restrict__ part, long long nxy, long long nv,
                              int groups) {
  const long long ixy = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int g = blockIdx.y;
  if (ixy >= nxy) return;
  const long long v0 = nv * g / groups, v1 = nv * (g + 1) / groups;
  double s = 0.0;
  const T *p = f + ixy + v0 * nxy;
#pragma unroll 8
  for (long long v = v0; v < v1; ++v, p += nxy) s += (double)__ldg(p);
  part[(long long)g * nxy + ixy] = s;
}

__global__ void __launch_bounds__(kMomentCells * kMomentSlices)
    k_rho_finish(const double *__restrict__ part, double *__restrict__ rho, long long nxy, int groups, double dvx,
                 double dvy) {
  moment_finish(part, rho, nxy, groups, dvx, dvy);
}

// ---- field_poisson pieces.
__global__ void k_rho_minus_one(double *__restrict__ rho, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) rho[i] -= 1.;
}

// field.cpp:48-63 (thrust variant): analytic fields of cases 2 and 6.
__global__ void k_analytic_field(double *__restrict__ ex, double *__restrict__ ey, int nx, int ny, int idcase,
                                 double minx, double miny, double dx, double dy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nx * ny) return;
  const int ix = i % nx, iy = i / nx;
  if (idcase == 2) {
    ex[i] = -(minx + ix * dx);
    ey[i] = 0.;
  } else {
    ey[i] = -(miny + iy * dy);
    ex[i] = 0.;
  }
}

// efield.cpp:68-99: the mode-wise solve (poisson.cuh) of every mode of the
// half spectrum, in place for phi_hat.
__global__ void k_poisson_solve(cufftDoubleComplex *__restrict__ rho_hat, cufftDoubleComplex *__restrict__ ex_hat,
                                cufftDoubleComplex *__restrict__ ey_hat, int nx1h, int nx2, double kx0,
                                double ky0, double normcoeff) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nx1h * nx2) return;
  const int ix1 = i % nx1h, ix2 = i / nx1h;
  const cufftDoubleComplex r = rho_hat[i];
  double2 e1, e2, r1;
  poisson_mode(ix1, ix2, nx2, make_double2(r.x, r.y), kx0, ky0, normcoeff, e1, e2, r1);
  ex_hat[i] = make_cuDoubleComplex(e1.x, e1.y);
  ey_hat[i] = make_cuDoubleComplex(e2.x, e2.y);
  rho_hat[i] = make_cuDoubleComplex(r1.x, r1.y);
}

// ---- Diags::compute: Kahan-compensated FP64 sums of rho and |E|^2 in one
// block, fixed order (deterministic).  diags.cpp:31-52 (OpenMP variant's
// mass formula sum*dx*dy; the thrust variant's `*= dx + dy` is a typo).
__device__ __forceinline__ void kahan_add(double &sum, double &c, double x) {
  const double y = x - c;
  const double t = sum + y;
  c = (t - sum) - y;
  sum = t;
}

__global__ void k_diags(const double *__restrict__ rho, const double *__restrict__ ex, const double *__restrict__ ey,
                        long long n, double dx, double dy, double *__restrict__ nrj_hist,
                        double *__restrict__ mass_hist, double *__restrict__ nrjx_hist,
                        double *__restrict__ nrjy_hist, int iter) {
  // Kahan sums of rho, Ex^2 + Ey^2, Ex^2, Ey^2.
  // Each thread's elements in order; the loads of four of them are issued
  // before their adds so that their latencies overlap.
  double s[4] = {0., 0., 0., 0.}, c[4] = {0., 0., 0., 0.};
  const long long step = blockDim.x;
  long long i = threadIdx.x;
  for (; i + 3 * step < n; i += 4 * step) {
    double r[4], a[4], b[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      r[u] = rho[i + u * step];
      a[u] = ex[i + u * step];
      b[u] = ey[i + u * step];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double ax = __dmul_rn(a[u], a[u]), by = __dmul_rn(b[u], b[u]);
      kahan_add(s[0], c[0], r[u]);
      kahan_add(s[1], c[1], __dadd_rn(ax, by));
      kahan_add(s[2], c[2], ax);
      kahan_add(s[3], c[3], by);
    }
  }
  for (; i < n; i += step) {
    const double a = ex[i], b = ey[i];
    const double ax = __dmul_rn(a, a), by = __dmul_rn(b, b);
    kahan_add(s[0], c[0], rho[i]);
    kahan_add(s[1], c[1], __dadd_rn(ax, by));
    kahan_add(s[2], c[2], ax);
    kahan_add(s[3], c[3], by);
  }
  __shared__ double ws[4][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double v = s[k] - c[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) ws[k][warp] = v;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    double v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = lane < nw ? ws[k][lane] : 0.;
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    }
    if (lane == 0) {
      double e = sqrt(v[1] * dx * dy);
      e = e > 1.e-30 ? log(e) : -1.e9;
      nrj_hist[iter] = e;
      mass_hist[iter] = v[0] * dx * dy;
      // miniapps/vlp4d_mpi/thrust/Diags.cpp:63-64.
      nrjx_hist[iter] = sqrt(0.5 * v[2] * dx * dy);
      nrjy_hist[iter] = sqrt(0.5 * v[3] * dx * dy);
    }
  }
}

// ---- L2 norm of f (miniapps/vlp4d_mpi/thrust/Diags.cpp:68-92):
// l2norm = sqrt(sum f^2 * dx dy dvx dvy).  Each block keeps Kahan sums per
// thread (grid-stride, 16-byte loads), reduces them in a fixed order and
// writes one (sum, compensation) pair; one block adds the pairs in order.
template <typename T>
__global__ void k_l2_partial(const T *__restrict__ f, long long n, double *__restrict__ part) {
  double sum = 0., comp = 0.;
  const long long n4 = n / 4;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    T v[4];
    load4(f + 4 * i, v);
#pragma unroll
    for (int k = 0; k < 4; ++k) kahan_add(sum, comp, (double)v[k] * (double)v[k]);
  }
  if (blockIdx.x == 0)
    for (long long i = 4 * n4 + threadIdx.x; i < n; i += blockDim.x) kahan_add(sum, comp, (double)f[i] * (double)f[i]);
  __shared__ double ws[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double v = sum - comp;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) ws[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s2 = 0., c2 = 0.;
    for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) kahan_add(s2, c2, ws[w]);
    part[2 * blockIdx.x] = s2;
    part[2 * blockIdx.x + 1] = c2;
  }
}

__global__ void k_l2_finish(const double *__restrict__ part, int blocks, double scale, double *__restrict__ out) {
  if (threadIdx.x != 0) return;
  double s = 0., c = 0.;
  for (int b = 0; b < blocks; ++b) {
    kahan_add(s, c, part[2 * b]);
    kahan_add(s, c, -part[2 * b + 1]);
  }
  *out = sqrt((s - c) * scale);
}

// ---- initcase.
template <typename T>
__global__ void k_init_case(T *__restrict__ f, Grid g, int ivy0, int ic, double amp, double k, double u) {
  const long long total = g.cells();
  const double PI = 3.14159265358979323846;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(idx % g.n[0]);
    long long r = idx / g.n[0];
    const int iy = (int)(r % g.n[1]);
    r /= g.n[1];
    const int ivx = (int)(r % g.n[2]);
    const int ivy = (int)(r / g.n[2]);
    const double x = g.minp[0] + ix * g.dx[0];
    const double y = g.minp[1] + iy * g.dx[1];
    const double vx = g.minp[2] + ivx * g.dx[2];
    const double vy = g.minp[3] + (ivy0 + ivy) * g.dx[3];  // ivy0: first owned plane of a slab
    double val = 0.;
    if (ic == VLP4D_IC_SLD10) {  // init.cpp:234-256
      val = (1. / (2 * PI)) * exp(-0.5 * (vx * vx + vy * vy)) * (1 + 0.05 * (cos(0.5 * x) * cos(0.5 * y)));
    } else if (ic == VLP4D_IC_TSI20) {  // init.cpp:258-285
      const double xi = 0.90, alpha = 0.05;
      val = (1 + alpha * (cos(0.5 * x))) * 1 / (2 * PI) * ((2 - 2 * xi) / (3 - 2 * xi)) *
            (1 + .5 * vx * vx / (1 - xi)) * exp(-.5 * (vx * vx + vy * vy));
    } else if (ic == VLP4D_IC_CYL02 || ic == VLP4D_IC_CYL05) {  // init.cpp:143-232
      const double PERIOD = 0.5 * PI, AMPLI = 4, cc = 0.50 * (6. / 16.), rc = 0.50 * (4. / 16.);
      const double xx = ic == VLP4D_IC_CYL02 ? x : y, vv = ic == VLP4D_IC_CYL02 ? vx : vy;
      double hv = 0.0, hx = 0.0;
      if ((vv <= cc + rc) && (vv >= cc - rc)) hv = cos(PERIOD * ((vv - cc) / rc));
      else if ((vv <= -cc + rc) && (vv >= -cc - rc)) hv = -cos(PERIOD * ((vv + cc) / rc));
      if ((xx <= cc + rc) && (xx >= cc - rc)) hx = cos(PERIOD * ((xx - cc) / rc));
      else if ((xx <= -cc + rc) && (xx >= -cc - rc)) hx = -cos(PERIOD * ((xx + cc) / rc));
      val = AMPLI * hx * hv;
    } else if (ic == VLP4D_IC_LANDAU_SUM) {
      val = (1. + amp * cos(k * x) + amp * cos(k * y)) * (exp(-0.5 * (vx * vx + vy * vy)) / (2 * PI));
    } else if (ic == VLP4D_IC_TWO_STREAM) {
      const double s = 1. / sqrt(2 * PI);
      const double mvy = s * exp(-0.5 * vy * vy);
      const double mb = 0.5 * (s * exp(-0.5 * (vx - u) * (vx - u)) + s * exp(-0.5 * (vx + u) * (vx + u)));
      val = (1. + amp * cos(k * x) + amp * cos(k * y)) * mb * mvy;
    }
    f[idx] = (T)val;
  }
}

// ---- 2D transpose (column-major rows x cols -> cols x rows) through a
// padded 32x32 shared tile: both the read and the write are coalesced.
template <typename E>
__global__ void k_transpose(const E *__restrict__ in, E *__restrict__ out, int rows, int cols) {
  __shared__ E tile[32][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = r0 + threadIdx.x, c = c0 + j;
    if (r < rows && c < cols) tile[j][threadIdx.x] = in[(long long)c * rows + r];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = c0 + threadIdx.x, r = r0 + j;
    if (r < rows && c < cols) out[(long long)r * cols + c] = tile[threadIdx.x][j];
  }
}

}  // namespace

int launch_field_rho(vlp4d_ctx *c, const void *fn, cudaStream_t s) {
  const long long nxy = c->g.nxy(), nv = c->g.nv();
  const int threads = 256;
  const int groups = c->rho_groups;
  dim3 grid((unsigned)((nxy + threads - 1) / threads), (unsigned)groups);
  if (c->dtype == VLP4D_F64)
    k_rho_partial<double><<<grid, threads, 0, s>>>((const double *)fn, c->rho_part, nxy, nv, groups);
  else
    k_rho_partial<float><<<grid, threads, 0, s>>>((const float *)fn, c->rho_part, nxy, nv, groups);
  VLP4D_LAUNCH_CHECK();
  return launch_rho_finish(c, groups, s);
}

int launch_rho_finish(vlp4d_ctx *c, int groups, cudaStream_t s) {
  const long long nxy = c->g.nxy();
  k_rho_finish<<<(unsigned)((nxy + kMomentCells - 1) / kMomentCells), kMomentCells * kMomentSlices, 0, s>>>(
      c->rho_part, c->rho, nxy, groups, c->g.dx[2], c->g.dx[3]);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

int launch_field_poisson(vlp4d_ctx *c, cudaStream_t s) {
  const int nx = c->g.n[0], ny = c->g.n[1];
  const long long n2 = (long long)nx * ny;
  const int threads = 256;
  const int idcase = c->dom.idcase;
  if (idcase == 2 || idcase == 6) {
    k_analytic_field<<<(unsigned)((n2 + threads - 1) / threads), threads, 0, s>>>(
        c->ex, c->ey, nx, ny, idcase, c->g.minp[0], c->g.minp[1], c->g.dx[0], c->g.dx[1]);
    VLP4D_LAUNCH_CHECK();
    return VLP4D_OK;
  }
  // Cases 10 and 20 solve for rho - 1 (field.cpp:65-72).
  const bool minus_one = idcase == 10 || idcase == 20;
  if (field_cluster_available(c)) return launch_field_cluster(c, minus_one ? 1. : 0., s);
  if (minus_one) {
    k_rho_minus_one<<<(unsigned)((n2 + threads - 1) / threads), threads, 0, s>>>(c->rho, n2);
    VLP4D_LAUNCH_CHECK();
  }
  VLP4D_CUFFT_TRY(cufftSetStream(c->plan_fwd, s));
  VLP4D_CUFFT_TRY(cufftSetStream(c->plan_bwd, s));
  VLP4D_CUFFT_TRY(cufftExecD2Z(c->plan_fwd, c->rho, c->rho_hat));
  const int nx1h = nx / 2 + 1;
  const double kx0 = 2 * M_PI / c->g.maxp[0];  // efield.cpp:44-45: 2*pi / maxPhy
  const double ky0 = 2 * M_PI / c->g.maxp[1];
  const double normcoeff = 1.0 / (double)(nx * ny);
  const int nh = nx1h * ny;
  k_poisson_solve<<<(nh + threads - 1) / threads, threads, 0, s>>>(c->rho_hat, c->ex_hat, c->ey_hat, nx1h, ny, kx0,
                                                                    ky0, normcoeff);
  VLP4D_LAUNCH_CHECK();
  // phi (into rho), ex, ey: one batched inverse transform over the three
  // spectra (slices of one allocation; the plan's input and output batch
  // distances are the spectrum and field slice strides).
  VLP4D_CUFFT_TRY(cufftSetStream(c->plan_bwd3, s));
  VLP4D_CUFFT_TRY(cufftExecZ2D(c->plan_bwd3, c->rho_hat, c->rho));
  return VLP4D_OK;
}

int launch_diags(vlp4d_ctx *c, int iter, cudaStream_t s) {
  k_diags<<<1, 1024, 0, s>>>(c->rho, c->ex, c->ey, c->g.nxy(), c->g.dx[0], c->g.dx[1], c->nrj, c->mass, c->nrjx,
                             c->nrjy, iter);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

int diags_async(vlp4d_ctx *c, int iter, cudaStream_t s) {
  VLP4D_CUDA_TRY(cudaEventRecord(c->ev_fork, s));
  VLP4D_CUDA_TRY(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
  int rc = launch_diags(c, iter, c->side);
  if (rc) return rc;
  VLP4D_CUDA_TRY(cudaEventRecord(c->ev_join, c->side));
  return VLP4D_OK;
}

int diags_join(vlp4d_ctx *c, cudaStream_t s) {
  VLP4D_CUDA_TRY(cudaStreamWaitEvent(s, c->ev_join, 0));
  return VLP4D_OK;
}

int launch_l2norm(vlp4d_ctx *c, const void *fn, int iter, cudaStream_t s) {
  const long long n = c->g.cells();
  if ((uintptr_t)fn % 16) return fail_msg(VLP4D_ERR_INVALID_ARG, "diags_l2norm: f must be 16-byte aligned");
  if (c->dtype == VLP4D_F64)
    k_l2_partial<double><<<c->l2_blocks, 512, 0, s>>>((const double *)fn, n, c->l2_part);
  else
    k_l2_partial<float><<<c->l2_blocks, 512, 0, s>>>((const float *)fn, n, c->l2_part);
  VLP4D_LAUNCH_CHECK();
  const double scale = c->g.dx[0] * c->g.dx[1] * c->g.dx[2] * c->g.dx[3];
  k_l2_finish<<<1, 32, 0, s>>>(c->l2_part, c->l2_blocks, scale, c->l2norm + iter);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

int launch_init_case(vlp4d_ctx *c, void *f, int ic, double amp, double k, double u, cudaStream_t s) {
  const int threads = 256;
  long long blocks = (c->g.cells() + threads - 1) / threads;
  if (blocks > (long long)c->num_sms * 32) blocks = (long long)c->num_sms * 32;
  if (c->dtype == VLP4D_F64)
    k_init_case<double><<<(unsigned)blocks, threads, 0, s>>>((double *)f, c->g, c->ivy0, ic, amp, k, u);
  else
    k_init_case<float><<<(unsigned)blocks, threads, 0, s>>>((float *)f, c->g, c->ivy0, ic, amp, k, u);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

int launch_transpose(const void *in, void *out, int rows, int cols, int elem, cudaStream_t s) {
  dim3 block(32, 8), grid((rows + 31) / 32, (cols + 31) / 32);
  if (elem == 4) k_transpose<float><<<grid, block, 0, s>>>((const float *)in, (float *)out, rows, cols);
  else if (elem == 8) k_transpose<double><<<grid, block, 0, s>>>((const double *)in, (double *)out, rows, cols);
  else k_transpose<double2><<<grid, block, 0, s>>>((const double2 *)in, (double2 *)out, rows, cols);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

// Self-test of the bounded waits: one thread waits on a barrier phase that
// nothing completes (no arrival, no copy), gives up after `limit` cycles and
// records the timeout in the context's error word, exactly as the fused
// kernels do when a copy does not land.
__global__ void k_wait_selftest(int *err, long long limit) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
    if (!mbar_wait_limit(&bar, 0, limit)) atomicExch(err, 1);
  }
}

int launch_wait_selftest(vlp4d_ctx *c, long long limit, cudaStream_t s) {
  k_wait_selftest<<<1, 32, 0, s>>>(c->d_err, limit);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

}  // namespace vlp4d
