// The vlp4d_mpi step for one process (miniapps/vlp4d_mpi, Timestep.hpp:34-97
// without LAG_ORDER: cubic B-spline interpolation), FP64.
//
// Arrays are the reference's halo-extended views (RealView4D with offsets,
// Init.cpp:333-343): extents n[d] + 6 in every dimension, first index -3
// (HALO_PTS = 3), layout_left.  The step:
//   halo fill     periodic images; the outermost layer holds the sums
//                 sum_{j=1..8} alpha^j f(...) that stand in for the rest of
//                 the periodic line (Communication.hpp:756-896)
//   spline xy     cubic B-spline prefilter along x, then y (Spline.hpp:114-198)
//   advect 2D     x, y shift by dt/2 through the 4x4 spline (Advection.hpp
//                 thrust :95-226); only its velocity moment is used
//   field         rho, Poisson solve (the context's FP64 cuFFT solver)
//   spline vxvy   the prefilter along vx, then vy (Spline.hpp:429-469)
//   advect 4D     predictor-corrector foot with the field interpolated by
//                 3-point Lagrange, then the 4^4 spline interpolation
//                 (Advection.hpp thrust :228-415)
//   field, diagnostics and L2 norm of the new state.
//
// Two families of kernels:
// * the reference-facing entry points (vlp4d_mpi_halo_fill, _spline_xy,
//   _spline_vxvy, _advect_2d, _advect_4d) run the reference's arithmetic in
//   its order with every product and sum rounded separately (no contracted
//   FMA, as the reference's x86-64 build computes), so they reproduce it bit
//   for bit;
// * vlp4d_mpi_step fuses the sequence into four passes over f: the x/y pass
//   builds each (vx, vy) plane's halo in shared memory, prefilters it,
//   writes its coefficients and evaluates the 2D advection straight into
//   the velocity moment; the vx and vy passes extend and prefilter the v
//   lines; the 4D pass interpolates and accumulates the moment and the L2
//   norm of the new state.  Its arithmetic uses FMA and its own summation
//   order: equal to the reference up to rounding.
#include <cmath>
#include <cstdlib>
#include <vector>

#include "internal.cuh"

namespace vlp4d {
namespace {

constexpr int kH = 3;     // HALO_PTS
constexpr int kMmax = 8;  // terms of a boundary sum (MMAX)

// Geometry of the halo-extended array.
struct HGrid {
  int n[4];
  long long e[4];  // n + 6
  long long s[4];  // strides: 1, e0, e0 e1, e0 e1 e2
  int is[4];       // the same strides as int (an array has fewer than 2^31 elements)
  double minp[4], maxp[4], dx[4], inv_dx[4];
  // Admissible feet of the 4D advection (Advection.hpp thrust :249-250):
  // [min + local_min*h - h, min + local_max*h + h] with local = 0..n-1.
  double lo[4], hi[4];
  // The clamp of the v feet, min + (max - min) (Advection.hpp thrust :307-308).
  double vtop[4];
  double alpha, beta, sqrt3;
  __host__ __device__ long long at(int x, int y, int vx, int vy) const {
    return (long long)(x + kH) + s[1] * (y + kH) + s[2] * (vx + kH) + s[3] * (vy + kH);
  }
  __host__ __device__ long long total() const { return e[0] * e[1] * e[2] * e[3]; }
};

HGrid make_hgrid(const vlp4d_ctx *c) {
  HGrid h;
  for (int k = 0; k < 4; ++k) {
    h.n[k] = c->g.n[k];
    h.e[k] = c->g.n[k] + 2 * kH;
    h.minp[k] = c->g.minp[k];
    h.maxp[k] = c->g.maxp[k];
    h.dx[k] = c->g.dx[k];
    h.inv_dx[k] = 1. / c->g.dx[k];
    h.lo[k] = c->g.minp[k] + 0 * c->g.dx[k] - c->g.dx[k];
    h.hi[k] = c->g.minp[k] + (c->g.n[k] - 1) * c->g.dx[k] + c->g.dx[k];
    h.vtop[k] = c->g.minp[k] + (c->g.maxp[k] - c->g.minp[k]);
  }
  h.s[0] = 1;
  h.s[1] = h.e[0];
  h.s[2] = h.e[0] * h.e[1];
  h.s[3] = h.s[2] * h.e[2];
  for (int k = 0; k < 4; ++k) h.is[k] = (int)h.s[k];
  // Spline.hpp:21,36-37: sqrt3 = sqrt(3), alpha = sqrt3 - 2,
  // beta = sqrt3 * (1 - alpha*alpha) (host IEEE arithmetic).
  h.sqrt3 = std::sqrt(3.0);
  h.alpha = h.sqrt3 - 2.;
  h.beta = h.sqrt3 * (1. - h.alpha * h.alpha);
  return h;
}

__device__ __forceinline__ int wrapi(int i, int n) { return ((i % n) + n) % n; }

// Separately rounded arithmetic (the reference's x86-64 build has no FMA).
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// 8-byte asynchronous global-to-shared copies (through L1), one commit group
// per call site, waited for before the data is read.
__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// ---------------------------------------------------------------------------
// Halo fill of one process (Communication.hpp:713-754 through the local
// copy; boundary_condition :756-896; point lists of listBoundary :128-440).
// A halo point whose coordinates all lie in [-2, n+1] takes the periodic
// image.  A point in the outermost layer (-3 or n+2) of the dimensions B
// takes sum_{j_k=1..MMAX, k in B} alpha^(sum j_k) f(r + sum_k s_k j_k e_k),
// s_k = -1 (left layer) or +1 (right), r_k = (c_k - s_k) mod n_k for k in B
// and c_k mod n_k otherwise, with the highest dimension of B in the outer
// loop and the powers of alpha built by repeated products, as the
// reference does.  Every grid dimension is at least MMAX + 2 = 10, so the
// sums read interior points only.
// The value of halo point c (not a grid point) of a halo-filled array.
__device__ double halo_value(const double *__restrict__ f, const HGrid &h, const int c[4]) {
  int B[4], sg[4], r[4], m = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (c[k] == -kH || c[k] == h.n[k] + kH - 1) {
      sg[k] = c[k] == -kH ? -1 : 1;
      B[m++] = k;
      r[k] = wrapi(c[k] - sg[k], h.n[k]);
    } else {
      sg[k] = 0;
      r[k] = wrapi(c[k], h.n[k]);
    }
  }
  if (m == 0) return f[h.at(r[0], r[1], r[2], r[3])];
  int j[4] = {1, 1, 1, 1};
  double w[4];
  w[m - 1] = h.alpha;
  for (int l = m - 2; l >= 0; --l) w[l] = mul(h.alpha, w[l + 1]);
  double sum = 0.;
  for (;;) {
    int p[4] = {r[0], r[1], r[2], r[3]};
    for (int l = 0; l < m; ++l) p[B[l]] += sg[B[l]] * j[l];
    sum = add(sum, mul(f[h.at(p[0], p[1], p[2], p[3])], w[0]));
    int l = 0;
    w[0] = mul(w[0], h.alpha);
    while (l < m && ++j[l] > kMmax) {
      j[l] = 1;
      ++l;
      if (l < m) w[l] = mul(w[l], h.alpha);
    }
    if (l == m) break;
    for (int q = l - 1; q >= 0; --q) w[q] = mul(h.alpha, w[q + 1]);
  }
  return sum;
}

// One block per extended (vx, vy) plane: a plane with vx, vy both grid
// coordinates has only its x/y ring (e0 e1 - n0 n1 points) in the halo,
// any other plane is halo throughout.  Halo points only read grid points,
// so the order of the writes does not matter.
__global__ void k_mpi_halo(double *__restrict__ f, HGrid h) {
  const long long planes = h.e[2] * h.e[3];
  const int e0 = (int)h.e[0], e1 = (int)h.e[1];
  const int ring = e0 * e1 - h.n[0] * h.n[1];
  for (long long pl = blockIdx.x; pl < planes; pl += gridDim.x) {
    const int cvx = (int)(pl % h.e[2]) - kH, cvy = (int)(pl / h.e[2]) - kH;
    const bool vin = cvx >= 0 && cvx < h.n[2] && cvy >= 0 && cvy < h.n[3];
    const int count = vin ? ring : e0 * e1;
    for (int t = threadIdx.x; t < count; t += blockDim.x) {
      int cx, cy;
      if (vin) {
        // The ring: rows -3..-1 and n1..n1+2 in full, then the six halo
        // columns of the interior rows.
        const int full = 2 * kH * e0;
        if (t < full) {
          const int rr = t / e0;
          cy = rr < kH ? rr - kH : h.n[1] + rr - kH;
          cx = t % e0 - kH;
        } else {
          const int u = t - full, k = u % (2 * kH);
          cy = u / (2 * kH);
          cx = k < kH ? k - kH : h.n[0] + k - kH;
        }
      } else {
        cx = t % e0 - kH;
        cy = t / e0 - kH;
      }
      const int c[4] = {cx, cy, cvx, cvy};
      f[h.at(cx, cy, cvx, cvy)] = halo_value(f, h, c);
    }
  }
}

// ---------------------------------------------------------------------------
// The prefilter of one extended line (Spline.hpp:114-198, LONG_ENOUGH_BUFFER
// form): e[0] and e[L+1] hold the boundary sums, e[1..L] the points -2..n+1
// (L = n + 4).  e[1..L] become the spline coefficients; e[0], e[L+1] stay.
//   causal:      t[0] = e[0] + e[1],  t[k] = e[1+k] + alpha t[k-1]
//   right end:   c[L] = sqrt3 (e[L+1] + sum_{k=0..L-1} alpha^k e[L-k])
//   anticausal:  c[i] = beta t[i-1] + alpha c[i+1]
// In place: t[k-1] is stored at e[k] once e[k] has been read.  EXACT runs
// the reference's order (right-end sum from the original values, products
// and sums rounded separately); otherwise the right-end sum is accumulated
// by Horner during the causal pass and products fuse with the sums.
template <bool EXACT>
__device__ __forceinline__ void spline_line(double *__restrict__ e, long long st, int L, double alpha, double beta,
                                            double sqrt3) {
  if (EXACT) {
    double acc = add(e[(long long)(L + 1) * st], e[(long long)L * st]);
    double ak = alpha;
    for (int k = 1; k < L; ++k) {
      acc = add(acc, mul(e[(long long)(L - k) * st], ak));
      ak = mul(ak, alpha);
    }
    double t = add(e[0], e[st]);
    e[st] = t;
    for (int k = 1; k < L - 1; ++k) {
      t = add(e[(long long)(1 + k) * st], mul(alpha, t));
      e[(long long)(1 + k) * st] = t;
    }
    double c = mul(acc, sqrt3);
    e[(long long)L * st] = c;
    for (int i = L - 1; i >= 1; --i) {
      c = add(mul(beta, e[(long long)i * st]), mul(alpha, c));
      e[(long long)i * st] = c;
    }
  } else {
    // Chunks of 8 positions: the next chunk's values are loaded (in program
    // order) before the current chunk's results are stored, so the loads
    // are in flight while the recursion runs.
    constexpr int C = 8;
    const double e1 = e[st];
    double t = e[0] + e1;
    double hsum = e1;  // Horner: sum_{i=1..L} alpha^(L-i) e[i]
    e[st] = t;
    double buf[C], nxt[C];
#pragma unroll
    for (int j = 0; j < C; ++j) buf[j] = 2 + j <= L - 1 ? e[(long long)(2 + j) * st] : 0.;
    for (int i = 2; i <= L - 1; i += C) {
#pragma unroll
      for (int j = 0; j < C; ++j) nxt[j] = i + C + j <= L - 1 ? e[(long long)(i + C + j) * st] : 0.;
#pragma unroll
      for (int j = 0; j < C; ++j) {
        if (i + j <= L - 1) {
          hsum = fma(hsum, alpha, buf[j]);
          t = fma(alpha, t, buf[j]);
          e[(long long)(i + j) * st] = t;
        }
      }
#pragma unroll
      for (int j = 0; j < C; ++j) buf[j] = nxt[j];
    }
    hsum = fma(hsum, alpha, e[(long long)L * st]);
    double c = (e[(long long)(L + 1) * st] + hsum) * sqrt3;
    e[(long long)L * st] = c;
    // Anticausal: c[i] = beta t[i-1] + alpha c[i+1], the beta products off
    // the chain.
#pragma unroll
    for (int j = 0; j < C; ++j) buf[j] = L - 1 - j >= 1 ? beta * e[(long long)(L - 1 - j) * st] : 0.;
    for (int i = L - 1; i >= 1; i -= C) {
#pragma unroll
      for (int j = 0; j < C; ++j) nxt[j] = i - C - j >= 1 ? beta * e[(long long)(i - C - j) * st] : 0.;
#pragma unroll
      for (int j = 0; j < C; ++j) {
        if (i - j >= 1) {
          c = fma(alpha, c, buf[j]);
          e[(long long)(i - j) * st] = c;
        }
      }
#pragma unroll
      for (int j = 0; j < C; ++j) buf[j] = nxt[j];
    }
  }
}

// Cubic B-spline weights at fractional offset w (Advection.hpp:127-144),
// in the reference's order of operations.
template <bool EXACT>
__device__ __forceinline__ void bspline_w(double w, double eta[4]) {
  if (EXACT) {
    const double e3 = mul(mul(mul(1. / 6., w), w), w);
    const double e0 = sub(add(1. / 6., mul(mul(0.5, w), sub(w, 1.))), e3);
    const double e2 = sub(add(w, e0), mul(2., e3));
    const double e1 = sub(sub(sub(1., e0), e2), e3);
    eta[0] = e0;
    eta[1] = e1;
    eta[2] = e2;
    eta[3] = e3;
  } else {
    const double e3 = (1. / 6.) * w * w * w;
    const double e0 = (1. / 6.) + 0.5 * w * (w - 1.) - e3;
    const double e2 = w + e0 - 2. * e3;
    eta[0] = e0;
    eta[1] = 1. - e0 - e2 - e3;
    eta[2] = e2;
    eta[3] = e3;
  }
}

}  // namespace
}  // namespace vlp4d

namespace vlp4d {
namespace {

// ---------------------------------------------------------------------------
// Plane kernels.  A (vx, vy) plane of the extended array lives in shared
// memory with an odd row stride P >= nx + 6 (row r = y + 3, column c = x + 3):
// a thread walking a row and its neighbour walking the next row then hit
// different banks.

// x lines of every row, then y lines of columns x in [-2, nx+1]
// (Spline.hpp:128-196: the row update covers all rows, the column update
// the columns istart..iend).
template <bool EXACT>
__device__ void plane_prefilter(double *pl, int P, const HGrid &h) {
  const int E1 = h.n[1] + 2 * kH, E0 = h.n[0] + 2 * kH;
  for (int r = threadIdx.x; r < E1; r += blockDim.x)
    spline_line<EXACT>(pl + (long long)r * P, 1, h.n[0] + 4, h.alpha, h.beta, h.sqrt3);
  __syncthreads();
  for (int c = 1 + threadIdx.x; c < E0 - 1; c += blockDim.x)
    spline_line<EXACT>(pl + c, P, h.n[1] + 4, h.alpha, h.beta, h.sqrt3);
  __syncthreads();
}

// Spline::computeCoeff_xy on every plane of a halo-filled array, in place,
// in the reference's arithmetic.
__global__ void __launch_bounds__(256) k_mpi_spline_xy(double *__restrict__ f, HGrid h, int P) {
  extern __shared__ __align__(16) double pl[];
  const int E0 = h.n[0] + 2 * kH, E1 = h.n[1] + 2 * kH;
  const long long planes = h.e[2] * h.e[3];
  for (long long p = blockIdx.x; p < planes; p += gridDim.x) {
    double *g = f + p * h.s[2];
    for (int r = threadIdx.y; r < E1; r += blockDim.y)
      for (int c = threadIdx.x; c < E0; c += blockDim.x) cp_async8(pl + r * P + c, g + (long long)r * E0 + c);
    cp_async_wait_all();
    __syncthreads();
    // plane_prefilter indexes threads linearly.
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    for (int r = tid; r < E1; r += nt) spline_line<true>(pl + (long long)r * P, 1, h.n[0] + 4, h.alpha, h.beta, h.sqrt3);
    __syncthreads();
    for (int c = 1 + tid; c < E0 - 1; c += nt) spline_line<true>(pl + c, P, h.n[1] + 4, h.alpha, h.beta, h.sqrt3);
    __syncthreads();
    for (int r = threadIdx.y; r < E1; r += blockDim.y)
      for (int c = threadIdx.x; c < E0; c += blockDim.x) g[(long long)r * E0 + c] = pl[r * P + c];
    __syncthreads();
  }
}

// The x, y halo of a plane whose interior rows 3..ny+2, columns 3..nx+2 are
// loaded: x extension of the interior rows, then y extension of every
// column (a corner then holds the y sum of x sums: the reference's double
// sum up to rounding).
__device__ void plane_extend(double *pl, int P, const HGrid &h) {
  const int nx = h.n[0], ny = h.n[1];
  const int E0 = nx + 2 * kH;
  for (int i = threadIdx.x; i < ny * 6; i += blockDim.x) {
    double *row = pl + (long long)(i / 6 + kH) * P;
    const int k = i % 6;
    double v;
    if (k == 0 || k == 5) {
      // left: sum_j alpha^j f(nx-2-j) (column nx+1-j); right: f(1+j) (column 4+j)
      double w = h.alpha, s = 0.;
      for (int j = 1; j <= kMmax; ++j) {
        s = fma(row[k == 0 ? nx + 1 - j : 4 + j], w, s);
        w *= h.alpha;
      }
      v = s;
      row[k == 0 ? 0 : nx + 5] = v;
    } else {
      // columns 1, 2 <- nx+1, nx+2 ; nx+3, nx+4 <- 3, 4
      const int dst = k <= 2 ? k : nx + k;  // k = 3, 4 -> nx+3, nx+4
      const int src = k <= 2 ? nx + k : k;
      row[dst] = row[src];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < E0 * 6; i += blockDim.x) {
    const int c = i / 6, k = i % 6;
    double *col = pl + c;
    if (k == 0 || k == 5) {
      double w = h.alpha, s = 0.;
      for (int j = 1; j <= kMmax; ++j) {
        s = fma(col[(long long)(k == 0 ? ny + 1 - j : 4 + j) * P], w, s);
        w *= h.alpha;
      }
      col[(long long)(k == 0 ? 0 : ny + 5) * P] = s;
    } else {
      const int dst = k <= 2 ? k : ny + k;
      const int src = k <= 2 ? ny + k : k;
      col[(long long)dst * P] = col[(long long)src * P];
    }
  }
  __syncthreads();
}

// The fused x/y pass of vlp4d_mpi_step.  Each CTA takes the interior
// (vx, vy) planes p = blockIdx.x, blockIdx.x + gridDim.x, ...: loads the
// plane's grid points from fn, builds its halo, prefilters it, writes the
// coefficients of the whole extended plane into cxy, and evaluates the 2D
// advection by dt (Advection.hpp thrust :131-214) at every grid point,
// adding it to the thread's moment accumulators, planes in a fixed order.
// Thread t owns the CPT cells of column t % nx, rows (t / nx) * CPT ..;
// it walks them with a sliding window of four x sums, so a cell costs
// about 4 shared-memory loads instead of 16.  The accumulators go to
// part[blockIdx.x][ix + nx*iy] at the end.  A foot outside the spline's
// range sets bit 2 of *err (the reference stops: "Time step is too
// large").
template <int CPT>
__global__ void __launch_bounds__(512) k_mpi_xy_pass(const double *__restrict__ fn, double *__restrict__ cxy,
                                                     HGrid h, int P, double dt, double *__restrict__ part,
                                                     int *__restrict__ err) {
  extern __shared__ __align__(16) double pl[];
  const int nx = h.n[0], ny = h.n[1], nvx = h.n[2];
  const int E0 = nx + 2 * kH, E1 = ny + 2 * kH;
  const int nxy = nx * ny;
  const long long planes = (long long)nvx * h.n[3];
  double acc[CPT];
#pragma unroll
  for (int k = 0; k < CPT; ++k) acc[k] = 0.;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  // This thread's strip of the 2D advection: column ix, rows iy0 .. iy0+CPT-1.
  const int ix = threadIdx.x % nx, iy0 = (threadIdx.x / nx) * CPT;
  const bool own = iy0 < ny;
  bool bad = false;
  for (long long p = blockIdx.x; p < planes; p += gridDim.x) {
    const int ivx = (int)(p % nvx), ivy = (int)(p / nvx);
    const double *src = fn + h.at(0, 0, ivx, ivy);
    for (int iy = warp; iy < ny; iy += nwarps)
      for (int ix = lane; ix < nx; ix += 32) cp_async8(pl + (iy + kH) * P + ix + kH, src + (long long)iy * E0 + ix);
    cp_async_wait_all();
    __syncthreads();
    plane_extend(pl, P, h);
    plane_prefilter<false>(pl, P, h);
    double *dst = cxy + h.at(-kH, -kH, ivx, ivy);
    for (int r = warp; r < E1; r += nwarps)
      for (int c = lane; c < E0; c += 32) dst[(long long)r * E0 + c] = pl[r * P + c];
    // 2D advection at the grid points of the plane, from the coefficients.
    // The shift (dt vx, dt vy) is the same for the whole plane: one cell
    // offset and one set of weights per direction (the reference evaluates
    // them per cell; they differ only by the rounding of x_i - dt vx).
    const double vx = h.minp[2] + ivx * h.dx[2], vy = h.minp[3] + ivy * h.dx[3];
    const double fx = -dt * vx * h.inv_dx[0], fy = -dt * vy * h.inv_dx[1];
    const int mx = (int)floor(fx), my = (int)floor(fy);
    if (mx < -1 || mx > 0 || my < -1 || my > 0) bad = true;  // i0 = ix + mx must stay in [-1, nx-1]
    double ex[4], ey[4];
    bspline_w<false>(fx - mx, ex);
    bspline_w<false>(fy - my, ey);
    if (!bad && own) {
      // x sums of rows iy0 + my - 1 + r (r = 0 .. CPT + 2), a window of four.
      const double *b = pl + (iy0 + my - 1 + kH) * P + (ix + mx - 1 + kH);
      double w0 = 0., w1 = 0., w2 = 0.;
#pragma unroll
      for (int r = 0; r < CPT + 3; ++r) {
        double w3 = 0.;
        if (iy0 + r - 3 < ny) {  // row needed by some cell of the strip
          const double *row = b + r * P;
          w3 = ex[0] * row[0] + ex[1] * row[1] + ex[2] * row[2] + ex[3] * row[3];
        }
        if (r >= 3) {
          const int j = r - 3;
          if (iy0 + j < ny) acc[j] += ey[0] * w0 + ey[1] * w1 + ey[2] * w2 + ey[3] * w3;
        }
        w0 = w1;
        w1 = w2;
        w2 = w3;
      }
    }
    __syncthreads();
  }
  if (bad) atomicOr(err, 2);
  if (own) {
#pragma unroll
    for (int j = 0; j < CPT; ++j)
      if (iy0 + j < ny) part[(long long)blockIdx.x * nxy + ix + (long long)nx * (iy0 + j)] = acc[j];
  }
}

// ---------------------------------------------------------------------------
// v lines.  A warp takes a tile of 32 lines along dimension `dim` (2: vx,
// 3: vy) at 32 consecutive x positions and one (y, o) pair (o: the other v
// coordinate, in [olo, olo + no)); lane l owns the line at x = x0 + l, kept
// in shared memory as [position][lane] (conflict-free).  `in` may be `out`
// (each line is read before it is written, by its own lane).  EXTEND: the line's
// grid points (positions 0..n-1) come from `in` and its halo is built here
// (periodic images, boundary sums); otherwise all n + 6 positions come from
// `in` as they are.  Lines with o in [flo, fhi] are prefiltered (the
// reference's column update skips the outermost layer of the first v
// dimension, Spline.hpp:164).  All n + 6 positions go to `out`.
template <bool EXTEND, bool EXACT>
__global__ void __launch_bounds__(128) k_mpi_vlines(const double *in, double *out, HGrid h,
                                                    int dim, int olo, int no, int flo, int fhi) {
  extern __shared__ __align__(16) double tiles[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int n = h.n[dim];
  const int E = n + 2 * kH;
  double *tile = tiles + (long long)warp * E * 32;
  const int odim = dim == 2 ? 3 : 2;
  const long long sl = h.s[dim], so = h.s[odim];
  const int xchunks = (int)((h.e[0] + 31) / 32);
  const long long ntiles = (long long)xchunks * h.e[1] * no;
  for (long long t = (long long)blockIdx.x * nwarps + warp; t < ntiles; t += (long long)gridDim.x * nwarps) {
    const int xc = (int)(t % xchunks);
    const long long r = t / xchunks;
    const int y = (int)(r % h.e[1]) - kH;
    const int o = (int)(r / h.e[1]) + olo;
    const int x = xc * 32 + lane - kH;
    const bool live = x < h.n[0] + kH;
    // Line base: position -3 of the line dimension.
    const long long base = (long long)(x + kH) + h.s[1] * (y + kH) + so * (o + kH);
    if (live) {
      if (EXTEND) {
        for (int i = 0; i < n; ++i) cp_async8(tile + (i + kH) * 32 + lane, in + base + (long long)(i + kH) * sl);
      } else {
        for (int i = 0; i < E; ++i) cp_async8(tile + i * 32 + lane, in + base + (long long)i * sl);
      }
    }
    cp_async_wait_all();
    __syncwarp();
    if (live) {
      double *col = tile + lane;
      if (EXTEND) {
        double wl = h.alpha, sL = 0., sR = 0.;
        for (int j = 1; j <= kMmax; ++j) {
          sL = fma(col[(n + 1 - j) * 32], wl, sL);
          sR = fma(col[(4 + j) * 32], wl, sR);
          wl *= h.alpha;
        }
        col[0] = sL;
        col[1 * 32] = col[(n + 1) * 32];
        col[2 * 32] = col[(n + 2) * 32];
        col[(n + 3) * 32] = col[3 * 32];
        col[(n + 4) * 32] = col[4 * 32];
        col[(n + 5) * 32] = sR;
      }
      if (o >= flo && o <= fhi) spline_line<EXACT>(col, 32, n + 4, h.alpha, h.beta, h.sqrt3);
      for (int i = 0; i < E; ++i) out[base + (long long)i * sl] = col[i * 32];
    }
    __syncwarp();
  }
}

}  // namespace
}  // namespace vlp4d

namespace vlp4d {
namespace {

// ---------------------------------------------------------------------------
// Advection::advect_2D_xy (thrust Advection.hpp:95-226, spline branch
// :175-206) in the reference's arithmetic: fn's grid points receive the
// 4x4 spline interpolation of the coefficients in tmp at
// (x - dt vx, y - dt vy).  A foot outside [xmin-1, xmax] (in cells) sets
// bit 2 of *err and the point receives 0.
__global__ void k_mpi_advect_2d(const double *__restrict__ tmp, double *__restrict__ fn, HGrid h, double dt,
                                int *__restrict__ err) {
  const long long cells = (long long)h.n[0] * h.n[1] * h.n[2] * h.n[3];
  bool bad = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cells;
       i += (long long)gridDim.x * blockDim.x) {
    long long r = i;
    const int ix = (int)(r % h.n[0]);
    r /= h.n[0];
    const int iy = (int)(r % h.n[1]);
    r /= h.n[1];
    const int ivx = (int)(r % h.n[2]);
    const int ivy = (int)(r / h.n[2]);
    const double x = add(h.minp[0], mul((double)ix, h.dx[0]));
    const double y = add(h.minp[1], mul((double)iy, h.dx[1]));
    const double vx = add(h.minp[2], mul((double)ivx, h.dx[2]));
    const double vy = add(h.minp[3], mul((double)ivy, h.dx[3]));
    const double fx = mul(sub(sub(x, mul(dt, vx)), h.minp[0]), h.inv_dx[0]);
    const double fy = mul(sub(sub(y, mul(dt, vy)), h.minp[1]), h.inv_dx[1]);
    const int i0 = (int)floor(fx), i1 = (int)floor(fy);
    double v = 0.;
    if (i0 < -1 || i0 > h.n[0] - 1 || i1 < -1 || i1 > h.n[1] - 1) {
      bad = true;
    } else {
      double ex[4], ey[4];
      bspline_w<true>(sub(fx, (double)i0), ex);
      bspline_w<true>(sub(fy, (double)i1), ey);
      for (int ky = 0; ky < 4; ++ky) {
        const double *row = tmp + h.at(i0 - 1, i1 - 1 + ky, ivx, ivy);
        double s = 0.;
        for (int kx = 0; kx < 4; ++kx) s = add(s, mul(ex[kx], row[kx]));
        v = add(v, mul(ey[ky], s));
      }
    }
    fn[h.at(ix, iy, ivx, ivy)] = v;
  }
  if (bad) atomicOr(err, 2);
}

// 3-point Lagrange weights (Advection.hpp thrust :29-34).
template <bool EXACT>
__device__ __forceinline__ void lag3w(double p, double c[3]) {
  if (EXACT) {
    c[0] = mul(mul(.5, sub(p, 1.)), sub(p, 2.));
    c[1] = mul(mul(-1., p), sub(p, 2.));
    c[2] = mul(mul(.5, p), sub(p, 1.));
  } else {
    c[0] = .5 * (p - 1.) * (p - 2.);
    c[1] = -p * (p - 2.);
    c[2] = .5 * p * (p - 1.);
  }
}

// computeFeet (thrust Advection.hpp:260-309): half-step predictor with the
// cell's own field, the field interpolated (periodic 3x3 Lagrange) at the
// predicted (x, y), then the full-step foot; vx, vy clamped to the domain.
// Returns the foot in grid units (xs - min) / h per dimension and whether
// it lies in the admissible range.
template <bool EXACT>
__device__ __forceinline__ bool foot4d(const HGrid &h, const double *__restrict__ ex, const double *__restrict__ ey,
                                       int ix, int iy, int ivx, int ivy, double dt, double g[4]) {
  const int nx = h.n[0], ny = h.n[1];
  double x, y, vx, vy, hdt = mul(0.5, dt);
  if (EXACT) {
    x = add(h.minp[0], mul((double)ix, h.dx[0]));
    y = add(h.minp[1], mul((double)iy, h.dx[1]));
    vx = add(h.minp[2], mul((double)ivx, h.dx[2]));
    vy = add(h.minp[3], mul((double)ivy, h.dx[3]));
  } else {
    x = h.minp[0] + ix * h.dx[0];
    y = h.minp[1] + iy * h.dx[1];
    vx = h.minp[2] + ivx * h.dx[2];
    vy = h.minp[3] + ivy * h.dx[3];
  }
  double t[2];
  if (EXACT) {
    t[0] = mul(h.inv_dx[0], sub(sub(x, mul(hdt, vx)), h.minp[0]));
    t[1] = mul(h.inv_dx[1], sub(sub(y, mul(hdt, vy)), h.minp[1]));
  } else {
    t[0] = h.inv_dx[0] * (x - hdt * vx - h.minp[0]);
    t[1] = h.inv_dx[1] * (y - hdt * vy - h.minp[1]);
  }
  int ip[2];
  double c[2][3];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    // The reference's (n + ipos + k) % n; a far-off predictor (a time step
    // the range check will reject) is kept inside the field by the clamp
    // and the non-negative modulo.
    ip[j] = (int)fmax(fmin(round(t[j]) - 1., 1e9), -1e9);
    lag3w<EXACT>(EXACT ? sub(t[j], (double)ip[j]) : t[j] - ip[j], c[j]);
  }
  double e1 = 0., e2 = 0.;
  const int r0 = wrapi(ip[0], nx), r1 = wrapi(ip[1], ny);
#pragma unroll
  for (int k1 = 0; k1 < 3; ++k1) {
    const int jy = r1 + k1 >= ny ? r1 + k1 - ny : r1 + k1;
#pragma unroll
    for (int k0 = 0; k0 < 3; ++k0) {
      const int jx = r0 + k0 >= nx ? r0 + k0 - nx : r0 + k0;
      const int q = jx + nx * jy;
      if (EXACT) {
        const double w = mul(c[0][k0], c[1][k1]);
        e1 = add(e1, mul(w, __ldg(ex + q)));
        e2 = add(e2, mul(w, __ldg(ey + q)));
      } else {
        const double w = c[0][k0] * c[1][k1];
        e1 = fma(w, __ldg(ex + q), e1);
        e2 = fma(w, __ldg(ey + q), e2);
      }
    }
  }
  double xs[4];
  if (EXACT) {
    const double vxh = sub(vx, mul(hdt, e1)), vyh = sub(vy, mul(hdt, e2));
    xs[0] = sub(x, mul(dt, vxh));
    xs[1] = sub(y, mul(dt, vyh));
    xs[2] = fmax(fmin(sub(vx, mul(dt, e1)), h.vtop[2]), h.minp[2]);
    xs[3] = fmax(fmin(sub(vy, mul(dt, e2)), h.vtop[3]), h.minp[3]);
  } else {
    xs[0] = x - dt * (vx - hdt * e1);
    xs[1] = y - dt * (vy - hdt * e2);
    xs[2] = fmax(fmin(vx - dt * e1, h.vtop[2]), h.minp[2]);
    xs[3] = fmax(fmin(vy - dt * e2, h.vtop[3]), h.minp[3]);
  }
  bool ok = true;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    ok &= !(xs[j] < h.lo[j] || xs[j] > h.hi[j]);
    g[j] = EXACT ? mul(h.inv_dx[j], sub(xs[j], h.minp[j])) : h.inv_dx[j] * (xs[j] - h.minp[j]);
  }
  return ok;
}

// interp_4d (thrust Advection.hpp:311-385, spline branch): 4^4 tensor
// B-spline interpolation of the coefficients c at the foot g (grid units).
template <bool EXACT>
__device__ __forceinline__ double interp4d(const HGrid &h, const double *__restrict__ c, const double g[4]) {
  int ip[4];
  double eta[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    ip[j] = (int)floor(g[j]);
    bspline_w<EXACT>(EXACT ? sub(g[j], (double)ip[j]) : g[j] - ip[j], eta[j]);
  }
  const double *b = c + h.at(ip[0] - 1, ip[1] - 1, ip[2] - 1, ip[3] - 1);
  double f1 = 0.;
#pragma unroll
  for (int k3 = 0; k3 < 4; ++k3) {
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
      double f2 = 0.;
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) {
        const double *row = b + k1 * h.s[1] + k2 * h.s[2] + k3 * h.s[3];
        if (EXACT) {
          double f3 = 0.;
#pragma unroll
          for (int k0 = 0; k0 < 4; ++k0) f3 = add(f3, mul(eta[0][k0], __ldg(row + k0)));
          f2 = add(f2, mul(f3, eta[1][k1]));
        } else {
          const double f3 = eta[0][0] * __ldg(row) + eta[0][1] * __ldg(row + 1) + eta[0][2] * __ldg(row + 2) +
                            eta[0][3] * __ldg(row + 3);
          f2 = fma(f3, eta[1][k1], f2);
        }
      }
      f1 = EXACT ? add(f1, mul(mul(f2, eta[2][k2]), eta[3][k3])) : fma(f2 * eta[2][k2], eta[3][k3], f1);
    }
  }
  return f1;
}

// Advection::advect_4D at the grid points: block (32 x, 8 y) of (ix, iy),
// blockIdx.z = plane group; a thread takes the planes p = z, z + G, ...
// (p = ivx + nvx*ivy).  MOMENT also accumulates the velocity moment
// (part[z][ix + nx*iy]) and, per block, the sum of squares of the new
// values (l2[block] as a (sum, 0) pair) for the field and the L2 norm.
template <bool EXACT, bool MOMENT>
__global__ void __launch_bounds__(256) k_mpi_advect_4d(const double *__restrict__ c, double *__restrict__ fn,
                                                       const double *__restrict__ ex, const double *__restrict__ ey,
                                                       HGrid h, double dt, double *__restrict__ part,
                                                       double *__restrict__ l2, int *__restrict__ err) {
  const int ix = blockIdx.x * 32 + threadIdx.x, iy = blockIdx.y * 8 + threadIdx.y;
  const int G = gridDim.z;
  const bool live = ix < h.n[0] && iy < h.n[1];
  const long long planes = (long long)h.n[2] * h.n[3];
  double acc = 0., sq = 0.;
  bool bad = false;
  if (live) {
    for (long long p = blockIdx.z; p < planes; p += G) {
      const int ivx = (int)(p % h.n[2]), ivy = (int)(p / h.n[2]);
      double g[4];
      double v = 0.;
      if (foot4d<EXACT>(h, ex, ey, ix, iy, ivx, ivy, dt, g)) {
        v = interp4d<EXACT>(h, c, g);
      } else {
        bad = true;
      }
      fn[h.at(ix, iy, ivx, ivy)] = v;
      if (MOMENT) {
        acc += v;
        sq = fma(v, v, sq);
      }
    }
  }
  if (bad) atomicOr(err, 2);
  if (MOMENT) {
    if (live) part[(long long)blockIdx.z * h.n[0] * h.n[1] + ix + (long long)h.n[0] * iy] = acc;
    // Block sum of sq in a fixed order.
    __shared__ double ws[8];
    const int tid = threadIdx.y * 32 + threadIdx.x;
    double v = sq;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) ws[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
      double s = 0.;
      for (int w = 0; w < 8; ++w) s += ws[w];
      const long long b = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
      l2[2 * b] = s;
      l2[2 * b + 1] = 0.;
    }
  }
}

// The fused step's 4D pass with R cells per thread at consecutive y (same
// x, vx, vy).  Block (32 x, 4 rows of R y), blockIdx.z = plane group as in
// k_mpi_advect_4d.  When the R feet share their x, vx and vy cells and
// their y cells are consecutive (all but a few per mille of the groups),
// the group reads each (vx, vy) slab's R + 3 rows of four x values once
// and applies every cell's own weights from registers: 64 (R + 3) / R
// loads per cell instead of 256.  Other groups interpolate cell by cell.
template <int R, bool UK3>
__global__ void __launch_bounds__(128, R <= 2 ? 3 : 2) k_mpi_advect_4d_rows(const double *__restrict__ c, double *__restrict__ fn,
                                                           const double *__restrict__ ex,
                                                           const double *__restrict__ ey, HGrid h, double dt,
                                                           double *__restrict__ part, double *__restrict__ l2,
                                                           int *__restrict__ err) {
  const int ix = blockIdx.x * 32 + threadIdx.x;
  const int iy0 = (blockIdx.y * blockDim.y + threadIdx.y) * R;
  const int G = gridDim.z;
  const long long planes = (long long)h.n[2] * h.n[3];
  const long long nx = h.n[0];
  double racc[R], sq = 0.;
#pragma unroll
  for (int q = 0; q < R; ++q) racc[q] = 0.;
  bool bad = false;
  if (ix < h.n[0] && iy0 < h.n[1]) {
    for (long long p = blockIdx.z; p < planes; p += G) {
      const int ivx = (int)(p % h.n[2]), ivy = (int)(p / h.n[2]);
      double g[R][4];
      bool ok[R];
      bool fast = true;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int iy = iy0 + q;
        ok[q] = iy < h.n[1] && foot4d<false>(h, ex, ey, ix, iy < h.n[1] ? iy : iy0, ivx, ivy, dt, g[q]);
        fast &= ok[q];
      }
      int ip[R][4];
#pragma unroll
      for (int q = 0; q < R; ++q)
#pragma unroll
        for (int j = 0; j < 4; ++j) ip[q][j] = (int)floor(g[q][j]);
#pragma unroll
      for (int q = 1; q < R; ++q)
        fast &= ip[q][0] == ip[0][0] && ip[q][2] == ip[0][2] && ip[q][3] == ip[0][3] && ip[q][1] == ip[0][1] + q;
      double val[R];
      if (fast) {
        double e0[R][4], e1[R][4], e2[R][4], e3[R][4];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          bspline_w<false>(g[q][0] - ip[q][0], e0[q]);
          bspline_w<false>(g[q][1] - ip[q][1], e1[q]);
          bspline_w<false>(g[q][2] - ip[q][2], e2[q]);
          bspline_w<false>(g[q][3] - ip[q][3], e3[q]);
          val[q] = 0.;
        }
        const double *b = c + h.at(ip[0][0] - 1, ip[0][1] - 1, ip[0][2] - 1, ip[0][3] - 1);
#pragma unroll(UK3 ? 4 : 1)
        for (int k3 = 0; k3 < 4; ++k3) {
          // The cells' k3 weights (a select chain when k3 is not a constant).
          double w3[R];
#pragma unroll
          for (int q = 0; q < R; ++q)
            w3[q] = k3 == 0 ? e3[q][0] : (k3 == 1 ? e3[q][1] : (k3 == 2 ? e3[q][2] : e3[q][3]));
#pragma unroll
          for (int k2 = 0; k2 < 4; ++k2) {
            const double *slab = b + k2 * h.s[2] + k3 * h.s[3];
            double s2[R];
#pragma unroll
            for (int q = 0; q < R; ++q) s2[q] = 0.;
#pragma unroll
            for (int r = 0; r < R + 3; ++r) {
              const double *row = slab + r * h.s[1];
              const double v0 = __ldg(row), v1 = __ldg(row + 1), v2 = __ldg(row + 2), v3 = __ldg(row + 3);
#pragma unroll
              for (int q = 0; q < R; ++q) {
                const int k1 = r - q;
                if (k1 >= 0 && k1 < 4) {
                  const double x = e0[q][0] * v0 + e0[q][1] * v1 + e0[q][2] * v2 + e0[q][3] * v3;
                  s2[q] = fma(x, e1[q][k1], s2[q]);
                }
              }
            }
#pragma unroll
            for (int q = 0; q < R; ++q) val[q] = fma(s2[q] * e2[q][k2], w3[q], val[q]);
          }
        }
      } else {
#pragma unroll
        for (int q = 0; q < R; ++q) {
          val[q] = 0.;
          if (iy0 + q < h.n[1]) {
            if (ok[q]) val[q] = interp4d<false>(h, c, g[q]);
            else bad = true;
          }
        }
      }
#pragma unroll
      for (int q = 0; q < R; ++q) {
        if (iy0 + q < h.n[1]) {
          fn[h.at(ix, iy0 + q, ivx, ivy)] = val[q];
          racc[q] += val[q];
          sq = fma(val[q], val[q], sq);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < R; ++q)
      if (iy0 + q < h.n[1]) part[(long long)blockIdx.z * nx * h.n[1] + ix + nx * (iy0 + q)] = racc[q];
  }
  if (bad) atomicOr(err, 2);
  // Block sum of sq in a fixed order.
  __shared__ double ws[4];
  const int tid = threadIdx.y * 32 + threadIdx.x;
  double v = sq;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((tid & 31) == 0) ws[tid >> 5] = v;
  __syncthreads();
  if (tid == 0) {
    double t = 0.;
    for (int w = 0; w < (int)(blockDim.x * blockDim.y) / 32; ++w) t += ws[w];
    const long long bl = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
    l2[2 * bl] = t;
    l2[2 * bl + 1] = 0.;
  }
}

// ---------------------------------------------------------------------------
// initcase of vlp4d_mpi (Init.cpp:126-277) on a halo array: the halo is
// zero, as after init() (Init.cpp:370-372); grid points get
//   10 SLD10: (1/2pi) exp(-(vx^2+vy^2)/2) (1 + 0.05 cos(x/2) cos(y/2))
//   20 TSI20: 1/(4 pi vthx vthy) (1 - ax sin(kx x) - ay sin(ky y))
//             [exp(-((vx-vd)/vthx)^2/2 - (vy/vthy)^2/2) + (vx+vd) term],
//             vd 2.4, vthx 1, vthy 0.5, ax 0.05, ay 0.25, kx = ky = 0.2
//   2, 5 CYL02 / CYL05: AMPLI hx hv with the cosine bumps of x, vx (2) or
//             y, vy (5); case 5 leaves the last vx, y and x index at 0, as
//             the reference's loops do (Init.cpp:198-202 stop before
//             local_nxmax).
__global__ void k_mpi_init_case(double *__restrict__ f, HGrid h, int idcase) {
  const long long total = h.total();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    long long r0 = i;
    int c[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      c[k] = (int)(r0 % h.e[k]) - kH;
      r0 /= h.e[k];
    }
    bool inside = true;
#pragma unroll
    for (int k = 0; k < 4; ++k) inside &= (c[k] >= 0 && c[k] < h.n[k]);
    double v = 0.;
    if (inside) {
      const double x = h.minp[0] + c[0] * h.dx[0], y = h.minp[1] + c[1] * h.dx[1];
      const double vx = h.minp[2] + c[2] * h.dx[2], vy = h.minp[3] + c[3] * h.dx[3];
      if (idcase == 10) {
        const double sum = vx * vx + vy * vy;
        v = (1. / (2 * M_PI)) * exp(-0.5 * sum) * (1 + 0.05 * (cos(0.5 * x) * cos(0.5 * y)));
      } else if (idcase == 20) {
        const double vd = 2.4, vthx = 1.0, vthy = 0.5, ax = 0.05, ay = 0.25, kx = 0.2, ky = 0.2;
        const double a = (vx - vd) / vthx, b = (vx + vd) / vthx, q = vy / vthy;
        v = 1. / (4 * M_PI * vthx * vthy) * (1 - ax * sin(kx * x) - ay * sin(ky * y)) *
            (exp(-.5 * (a * a + q * q)) + exp(-.5 * (b * b + q * q)));
      } else if (idcase == 2 || idcase == 5) {
        const bool skip = idcase == 5 && (c[2] == h.n[2] - 1 || c[1] == h.n[1] - 1 || c[0] == h.n[0] - 1);
        if (!skip) {
          const double PERIOD = 0.5 * M_PI, AMPLI = 4, cc = 0.50 * (6. / 16.), rc = 0.50 * (4. / 16.);
          const double xx = idcase == 2 ? x : y, vv = idcase == 2 ? vx : vy;
          double hv = 0.0, hx = 0.0;
          if ((vv <= cc + rc) && (vv >= cc - rc)) hv = cos(PERIOD * ((vv - cc) / rc));
          else if ((vv <= -cc + rc) && (vv >= -cc - rc)) hv = -cos(PERIOD * ((vv + cc) / rc));
          if ((xx <= cc + rc) && (xx >= cc - rc)) hx = cos(PERIOD * ((xx - cc) / rc));
          else if ((xx <= -cc + rc) && (xx >= -cc - rc)) hx = -cos(PERIOD * ((xx + cc) / rc));
          v = AMPLI * hx * hv;
        }
      }
    }
    f[i] = v;
  }
}

// ---------------------------------------------------------------------------
// Velocity moment of the grid points of a halo array (Field.cpp:5-55):
// part[group][ixy] over the planes of the group.
__global__ void k_mpi_rho_partial(const double *__restrict__ f, double *__restrict__ part, HGrid h, int groups) {
  const long long nxy = (long long)h.n[0] * h.n[1];
  const long long ixy = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int g = blockIdx.y;
  if (ixy >= nxy) return;
  const int ix = (int)(ixy % h.n[0]), iy = (int)(ixy / h.n[0]);
  const long long nv = (long long)h.n[2] * h.n[3];
  const long long v0 = nv * g / groups, v1 = nv * (g + 1) / groups;
  double s = 0.;
  for (long long v = v0; v < v1; ++v) s += __ldg(f + h.at(ix, iy, (int)(v % h.n[2]), (int)(v / h.n[2])));
  part[(long long)g * nxy + ixy] = s;
}

__device__ __forceinline__ void kahan(double &s, double &c, double x) {
  const double y = x - c;
  const double t = s + y;
  c = (t - s) - y;
  s = t;
}

// Sum of squares of the grid points of a halo array, per block as a Kahan
// (sum, compensation) pair, threads reduced in a fixed order.
__global__ void __launch_bounds__(256) k_mpi_l2_partial(const double *__restrict__ f, HGrid h,
                                                        double *__restrict__ l2) {
  // A warp walks rows (32 x positions at a time); the block's 8 warps take
  // rows r = 8 * blockIdx + warp, stepping by 8 * gridDim.
  const long long rows = (long long)h.n[1] * h.n[2] * h.n[3];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double s = 0., cp = 0.;
  for (long long r = (long long)blockIdx.x * nw + warp; r < rows; r += (long long)gridDim.x * nw) {
    const int iy = (int)(r % h.n[1]);
    const long long rv = r / h.n[1];
    const double *row = f + h.at(0, iy, (int)(rv % h.n[2]), (int)(rv / h.n[2]));
    for (int ix = lane; ix < h.n[0]; ix += 32) {
      const double v = __ldg(row + ix);
      kahan(s, cp, v * v);
    }
  }
  __shared__ double ws[256];
  ws[threadIdx.x] = s - cp;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0., b = 0.;
    for (int t = 0; t < (int)blockDim.x; ++t) kahan(a, b, ws[t]);
    l2[2 * blockIdx.x] = a;
    l2[2 * blockIdx.x + 1] = b;
  }
}

// l2norm[iter] = sqrt(sum * dx dy dvx dvy) from `blocks` (sum, comp) pairs
// added in order (Diags.cpp:50-76).
__global__ void k_mpi_l2_finish(const double *__restrict__ l2, long long blocks, double scale,
                                double *__restrict__ out) {
  if (threadIdx.x != 0) return;
  double s = 0., c = 0.;
  for (long long b = 0; b < blocks; ++b) {
    kahan(s, c, l2[2 * b]);
    kahan(s, c, -l2[2 * b + 1]);
  }
  *out = sqrt(s * scale);
}

}  // namespace
}  // namespace vlp4d

// ---------------------------------------------------------------------------
// Host side.
namespace vlp4d {
namespace {

int mpi_check(const vlp4d_ctx *c, const char *what) {
  if (!c) return fail_msg(VLP4D_ERR_INVALID_ARG, std::string(what) + ": context is NULL");
  if (c->slab)
    return fail_msg(VLP4D_ERR_UNSUPPORTED, std::string(what) + ": the vlp4d_mpi arrays need an ordinary context");
  if (c->dtype != VLP4D_F64)
    return fail_msg(VLP4D_ERR_UNSUPPORTED, std::string(what) + ": the vlp4d_mpi path is FP64 (as the reference)");
  for (int k = 0; k < 4; ++k)
    if (c->g.n[k] < kMmax + 2)
      return fail_msg(VLP4D_ERR_INVALID_ARG,
                      std::string(what) + ": every grid dimension must be at least 10 (MMAX + 2, Init.cpp:85-89)");
  return VLP4D_OK;
}

int mpi_check_ptr(const void *p, const char *what) {
  if (!p) return fail_msg(VLP4D_ERR_INVALID_ARG, std::string(what) + ": array is NULL");
  if ((uintptr_t)p % 16) return fail_msg(VLP4D_ERR_INVALID_ARG, std::string(what) + ": array must be 16-byte aligned");
  return VLP4D_OK;
}

// Odd row stride of a shared-memory plane and its size in bytes.
int plane_stride(const HGrid &h) { return (int)(h.e[0] | 1); }
size_t plane_bytes(const HGrid &h) { return sizeof(double) * (size_t)h.e[1] * (size_t)plane_stride(h); }

int smem_limit(const vlp4d_ctx *c) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  return v;
}

int launch_halo(vlp4d_ctx *c, const HGrid &h, double *f, cudaStream_t s) {
  long long grid = (long long)c->num_sms * 8;
  if (grid > h.e[2] * h.e[3]) grid = h.e[2] * h.e[3];
  k_mpi_halo<<<(unsigned)grid, 256, 0, s>>>(f, h);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

int launch_spline_xy_exact(vlp4d_ctx *c, const HGrid &h, double *f, cudaStream_t s) {
  const size_t smem = plane_bytes(h);
  if (smem > (size_t)smem_limit(c))
    return fail_msg(VLP4D_ERR_UNSUPPORTED, "mpi_spline_xy: the (x, y) plane does not fit in shared memory");
  VLP4D_CUDA_TRY(cudaFuncSetAttribute(k_mpi_spline_xy, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  VLP4D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mpi_spline_xy, 256, smem));
  long long grid = (long long)c->num_sms * (per_sm > 0 ? per_sm : 1);
  const long long planes = h.e[2] * h.e[3];
  if (grid > planes) grid = planes;
  k_mpi_spline_xy<<<(unsigned)grid, dim3(32, 8), smem, s>>>(f, h, plane_stride(h));
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

// v lines along `dim` for o in [olo, olo + no), prefiltered for o in
// [flo, fhi].
template <bool EXTEND, bool EXACT>
int launch_vlines(vlp4d_ctx *c, const HGrid &h, const double *in, double *out, int dim, int olo, int no, int flo,
                  int fhi, cudaStream_t s) {
  const size_t tile = sizeof(double) * 32 * (size_t)h.e[dim];
  const int lim = smem_limit(c);
  int warps = (int)(lim / tile);
  if (warps > 4) warps = 4;
  if (warps < 1) return fail_msg(VLP4D_ERR_UNSUPPORTED, "mpi v lines: a tile does not fit in shared memory");
  const size_t smem = tile * warps;
  auto k = k_mpi_vlines<EXTEND, EXACT>;
  VLP4D_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  VLP4D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 32 * warps, smem));
  const long long tiles = (h.e[0] + 31) / 32 * h.e[1] * no;
  long long grid = (long long)c->num_sms * (per_sm > 0 ? per_sm : 1);
  const long long need = (tiles + warps - 1) / warps;
  if (grid > need) grid = need;
  k<<<(unsigned)grid, 32 * warps, smem, s>>>(in, out, h, dim, olo, no, flo, fhi);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

int launch_spline_vxvy_exact(vlp4d_ctx *c, const HGrid &h, double *f, cudaStream_t s) {
  int rc = launch_vlines<false, true>(c, h, f, f, 2, -kH, h.n[3] + 2 * kH, -kH, h.n[3] + kH - 1, s);
  if (rc) return rc;
  return launch_vlines<false, true>(c, h, f, f, 3, -kH + 1, h.n[2] + 4, -kH + 1, h.n[2] + kH - 2, s);
}

template <int CPT>
int launch_xy_pass_cpt(vlp4d_ctx *c, const HGrid &h, const double *fn, double *cxy, double dt, int *groups,
                       cudaStream_t s) {
  const size_t smem = plane_bytes(h);
  auto k = k_mpi_xy_pass<CPT>;
  VLP4D_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  VLP4D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 512, smem));
  long long grid = (long long)c->num_sms * (per_sm > 0 ? per_sm : 1);
  const long long planes = (long long)h.n[2] * h.n[3];
  if (grid > planes) grid = planes;
  if (grid > c->rho_part_groups) grid = c->rho_part_groups;
  k<<<(unsigned)grid, 512, smem, s>>>(fn, cxy, h, plane_stride(h), dt, c->rho_part, c->d_err);
  VLP4D_LAUNCH_CHECK();
  *groups = (int)grid;
  return VLP4D_OK;
}

// The fused x/y pass: fn's grid points -> coefficients of the extended
// (x, y) planes in cxy (interior v planes) and the moment partials of the
// 2D advection by dt.
int launch_xy_pass(vlp4d_ctx *c, const HGrid &h, const double *fn, double *cxy, double dt, int *groups,
                   cudaStream_t s) {
  if (plane_bytes(h) > (size_t)smem_limit(c))
    return fail_msg(VLP4D_ERR_UNSUPPORTED, "mpi_step: the (x, y) plane does not fit in shared memory");
  // Cells per thread: the smallest CPT whose strips (nx columns of
  // ceil(ny / CPT) strips) fit in the 512 threads.
  const long long nx = h.n[0], ny = h.n[1];
  auto fits = [&](long long cpt) { return nx * ((ny + cpt - 1) / cpt) <= 512; };
  if (nx > 512) return fail_msg(VLP4D_ERR_UNSUPPORTED, "mpi_step: nx above 512");
  if (fits(1)) return launch_xy_pass_cpt<1>(c, h, fn, cxy, dt, groups, s);
  if (fits(2)) return launch_xy_pass_cpt<2>(c, h, fn, cxy, dt, groups, s);
  if (fits(4)) return launch_xy_pass_cpt<4>(c, h, fn, cxy, dt, groups, s);
  if (fits(8)) return launch_xy_pass_cpt<8>(c, h, fn, cxy, dt, groups, s);
  if (fits(16)) return launch_xy_pass_cpt<16>(c, h, fn, cxy, dt, groups, s);
  if (fits(32)) return launch_xy_pass_cpt<32>(c, h, fn, cxy, dt, groups, s);
  return fail_msg(VLP4D_ERR_UNSUPPORTED, "mpi_step: the x/y plane needs more than 32 cells per thread");
}

// 4D advection of the coefficients c4 into fn's grid points; MOMENT: with
// the moment partials (groups written to *groups) and per-block sums of
// squares (*blocks pairs in c->mpi_part).
template <bool EXACT, bool MOMENT>
int launch_advect_4d(vlp4d_ctx *c, const HGrid &h, const double *c4, double *fn, double dt, int *groups,
                     long long *blocks, cudaStream_t s) {
  const dim3 block(32, 8);
  const long long bx = (h.n[0] + 31) / 32, by = (h.n[1] + 7) / 8;
  const long long planes = (long long)h.n[2] * h.n[3];
  // One resident wave (see launch_advect_4d_rows_r).
  int per_sm = 0;
  VLP4D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mpi_advect_4d<EXACT, MOMENT>, 256, 0));
  long long G = ((long long)c->num_sms * (per_sm > 0 ? per_sm : 1)) / (bx * by);
  if (G < 1) G = 1;
  if (G > planes) G = planes;
  if (MOMENT) {
    if (G > c->rho_part_groups) G = c->rho_part_groups;
    if (G * bx * by > c->mpi_part_cap) G = c->mpi_part_cap / (bx * by);
    if (G < 1) return fail_msg(VLP4D_ERR_UNSUPPORTED, "mpi 4D advection: too many (x, y) blocks for the partials");
  }
  const dim3 grid((unsigned)bx, (unsigned)by, (unsigned)G);
  k_mpi_advect_4d<EXACT, MOMENT><<<grid, block, 0, s>>>(c4, fn, c->ex, c->ey, h, dt, c->rho_part, c->mpi_part,
                                                         c->d_err);
  VLP4D_LAUNCH_CHECK();
  if (groups) *groups = (int)G;
  if (blocks) *blocks = G * bx * by;
  return VLP4D_OK;
}

template <int R, bool UK3>
int launch_advect_4d_rows_r(vlp4d_ctx *c, const HGrid &h, const double *c4, double *fn, double dt, int *groups,
                            long long *blocks, cudaStream_t s) {
  const dim3 block(32, 4);
  const long long bx = (h.n[0] + 31) / 32, by = (h.n[1] + 4 * R - 1) / (4 * R);
  const long long planes = (long long)h.n[2] * h.n[3];
  // One resident wave: every block walks the planes p = z, z + G, ... at
  // the same pace, so the blocks in flight read neighbouring (vx, vy)
  // slabs and the coefficients come from DRAM about once.
  int per_sm = 0;
  VLP4D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mpi_advect_4d_rows<R, UK3>, 128, 0));
  long long G = ((long long)c->num_sms * (per_sm > 0 ? per_sm : 1)) / (bx * by);
  if (G < 1) G = 1;
  if (G > planes) G = planes;
  if (G > c->rho_part_groups) G = c->rho_part_groups;
  if (G * bx * by > c->mpi_part_cap) G = c->mpi_part_cap / (bx * by);
  if (G < 1) return fail_msg(VLP4D_ERR_UNSUPPORTED, "mpi 4D advection: too many (x, y) blocks for the partials");
  k_mpi_advect_4d_rows<R, UK3><<<dim3((unsigned)bx, (unsigned)by, (unsigned)G), block, 0, s>>>(
      c4, fn, c->ex, c->ey, h, dt, c->rho_part, c->mpi_part, c->d_err);
  VLP4D_LAUNCH_CHECK();
  *groups = (int)G;
  *blocks = G * bx * by;
  return VLP4D_OK;
}

// Cells per thread of the fused 4D pass (VLP4D_MPI_ROWS = 1..4 overrides;
// 1 is the cell-per-thread kernel).
int mpi_rows() {
  static int r = [] {
    const char *e = getenv("VLP4D_MPI_ROWS");
    const int v = e && *e ? atoi(e) : 2;
    return v >= 1 && v <= 4 ? v : 2;
  }();
  return r;
}

// Whether the fused 4D pass unrolls its k3 loop (VLP4D_MPI_UNROLL = 0/1;
// unrolled: more loads in flight, more registers).
bool mpi_unroll_k3() {
  static bool u = [] {
    const char *e = getenv("VLP4D_MPI_UNROLL");
    return e && *e ? atoi(e) != 0 : true;
  }();
  return u;
}

int launch_advect_4d_fused(vlp4d_ctx *c, const HGrid &h, const double *c4, double *fn, double dt, int *groups,
                           long long *blocks, cudaStream_t s) {
  const bool u = mpi_unroll_k3();
  switch (mpi_rows()) {
    case 2:
      return u ? launch_advect_4d_rows_r<2, true>(c, h, c4, fn, dt, groups, blocks, s)
               : launch_advect_4d_rows_r<2, false>(c, h, c4, fn, dt, groups, blocks, s);
    case 3:
      return u ? launch_advect_4d_rows_r<3, true>(c, h, c4, fn, dt, groups, blocks, s)
               : launch_advect_4d_rows_r<3, false>(c, h, c4, fn, dt, groups, blocks, s);
    case 4:
      return u ? launch_advect_4d_rows_r<4, true>(c, h, c4, fn, dt, groups, blocks, s)
               : launch_advect_4d_rows_r<4, false>(c, h, c4, fn, dt, groups, blocks, s);
    default: return launch_advect_4d<false, true>(c, h, c4, fn, dt, groups, blocks, s);
  }
}

int launch_rho_halo(vlp4d_ctx *c, const HGrid &h, const double *f, cudaStream_t s) {
  const long long nxy = (long long)h.n[0] * h.n[1];
  const int groups = c->rho_groups;
  k_mpi_rho_partial<<<dim3((unsigned)((nxy + 255) / 256), groups), 256, 0, s>>>(f, c->rho_part, h, groups);
  VLP4D_LAUNCH_CHECK();
  return launch_rho_finish(c, groups, s);
}

int launch_l2_halo(vlp4d_ctx *c, const HGrid &h, const double *f, int iter, cudaStream_t s) {
  long long blocks = (long long)c->num_sms * 4;
  if (blocks > c->mpi_part_cap) blocks = c->mpi_part_cap;
  k_mpi_l2_partial<<<(unsigned)blocks, 256, 0, s>>>(f, h, c->mpi_part);
  VLP4D_LAUNCH_CHECK();
  const double scale = h.dx[0] * h.dx[1] * h.dx[2] * h.dx[3];
  k_mpi_l2_finish<<<1, 32, 0, s>>>(c->mpi_part, blocks, scale, c->l2norm + iter);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

}  // namespace
}  // namespace vlp4d

using namespace vlp4d;

extern "C" {

size_t vlp4d_mpi_size(const vlp4d_ctx *ctx) {
  if (!ctx) return 0;
  size_t n = 1;
  for (int k = 0; k < 4; ++k) n *= (size_t)(ctx->g.n[k] + 2 * kH);
  return n;
}

int vlp4d_mpi_init_case(vlp4d_ctx *ctx, void *fn, void *stream) {
  int rc = mpi_check(ctx, "mpi_init_case");
  if (rc || (rc = mpi_check_ptr(fn, "mpi_init_case"))) return rc;
  const int ic = ctx->dom.idcase;
  if (ic != 2 && ic != 5 && ic != 10 && ic != 20)
    return fail_msg(VLP4D_ERR_INVALID_ARG, "mpi_init_case: unknown test case (the reference aborts, Init.cpp:142-145)");
  k_mpi_init_case<<<ctx->num_sms * 8, 256, 0, (cudaStream_t)stream>>>((double *)fn, make_hgrid(ctx), ic);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

int vlp4d_mpi_halo_fill(vlp4d_ctx *ctx, void *fn, void *stream) {
  int rc = mpi_check(ctx, "mpi_halo_fill");
  if (rc || (rc = mpi_check_ptr(fn, "mpi_halo_fill"))) return rc;
  return launch_halo(ctx, make_hgrid(ctx), (double *)fn, (cudaStream_t)stream);
}

int vlp4d_mpi_spline_xy(vlp4d_ctx *ctx, void *fn, void *stream) {
  int rc = mpi_check(ctx, "mpi_spline_xy");
  if (rc || (rc = mpi_check_ptr(fn, "mpi_spline_xy"))) return rc;
  return launch_spline_xy_exact(ctx, make_hgrid(ctx), (double *)fn, (cudaStream_t)stream);
}

int vlp4d_mpi_spline_vxvy(vlp4d_ctx *ctx, void *fn, void *stream) {
  int rc = mpi_check(ctx, "mpi_spline_vxvy");
  if (rc || (rc = mpi_check_ptr(fn, "mpi_spline_vxvy"))) return rc;
  return launch_spline_vxvy_exact(ctx, make_hgrid(ctx), (double *)fn, (cudaStream_t)stream);
}

int vlp4d_mpi_advect_2d(vlp4d_ctx *ctx, void *fn, void *fn_tmp, double dt, void *stream) {
  int rc = mpi_check(ctx, "mpi_advect_2d");
  if (rc || (rc = mpi_check_ptr(fn, "mpi_advect_2d")) || (rc = mpi_check_ptr(fn_tmp, "mpi_advect_2d"))) return rc;
  if (fn == fn_tmp) return fail_msg(VLP4D_ERR_INVALID_ARG, "mpi_advect_2d: fn and fn_tmp must differ");
  const HGrid h = make_hgrid(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  VLP4D_CUDA_TRY(cudaMemcpyAsync(fn_tmp, fn, sizeof(double) * (size_t)h.total(), cudaMemcpyDeviceToDevice, s));
  k_mpi_advect_2d<<<ctx->num_sms * 8, 256, 0, s>>>((const double *)fn_tmp, (double *)fn, h, dt, ctx->d_err);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

int vlp4d_mpi_advect_4d(vlp4d_ctx *ctx, void *fn, void *tmp_fn, double dt, void *stream) {
  int rc = mpi_check(ctx, "mpi_advect_4d");
  if (rc || (rc = mpi_check_ptr(fn, "mpi_advect_4d")) || (rc = mpi_check_ptr(tmp_fn, "mpi_advect_4d"))) return rc;
  if (fn == tmp_fn) return fail_msg(VLP4D_ERR_INVALID_ARG, "mpi_advect_4d: fn and tmp_fn must differ");
  const HGrid h = make_hgrid(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  VLP4D_CUDA_TRY(cudaMemcpyAsync(tmp_fn, fn, sizeof(double) * (size_t)h.total(), cudaMemcpyDeviceToDevice, s));
  return launch_advect_4d<true, false>(ctx, h, (const double *)tmp_fn, (double *)fn, dt, nullptr, nullptr, s);
}

int vlp4d_mpi_field(vlp4d_ctx *ctx, const void *fn, void *stream) {
  int rc = mpi_check(ctx, "mpi_field");
  if (rc || (rc = mpi_check_ptr(fn, "mpi_field"))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if ((rc = launch_rho_halo(ctx, make_hgrid(ctx), (const double *)fn, s))) return rc;
  return launch_field_poisson(ctx, s);
}

int vlp4d_mpi_l2norm(vlp4d_ctx *ctx, const void *fn, int iter, void *stream) {
  int rc = mpi_check(ctx, "mpi_l2norm");
  if (rc || (rc = mpi_check_ptr(fn, "mpi_l2norm"))) return rc;
  if (iter < 0 || iter >= ctx->hist_len) return fail_msg(VLP4D_ERR_INVALID_ARG, "mpi_l2norm: iter outside [0, nbiter]");
  return launch_l2_halo(ctx, make_hgrid(ctx), (const double *)fn, iter, (cudaStream_t)stream);
}

int vlp4d_mpi_step(vlp4d_ctx *ctx, void *fn, void *fnp1, int iter, void *stream) {
  int rc = mpi_check(ctx, "mpi_step");
  if (rc || (rc = mpi_check_ptr(fn, "mpi_step")) || (rc = mpi_check_ptr(fnp1, "mpi_step"))) return rc;
  if (fn == fnp1) return fail_msg(VLP4D_ERR_INVALID_ARG, "mpi_step: fn and fnp1 must differ");
  if (iter < 0 || iter >= ctx->hist_len) return fail_msg(VLP4D_ERR_INVALID_ARG, "mpi_step: iter outside [0, nbiter]");
  const HGrid h = make_hgrid(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  double *f = (double *)fn, *g = (double *)fnp1;
  const double dt = ctx->dom.dt;
  int groups = 0;
  // x/y: f's grid points -> x/y coefficients of the interior v planes (in g)
  // and the moment of the half-step 2D advection.
  if ((rc = launch_xy_pass(ctx, h, f, g, 0.5 * dt, &groups, s))) return rc;
  if ((rc = launch_rho_finish(ctx, groups, s))) return rc;
  if ((rc = launch_field_poisson(ctx, s))) return rc;
  // vx lines of the interior vy planes (g -> f), then vy lines of every vx
  // position (in place in f): f holds the 4D coefficients.
  if ((rc = launch_vlines<true, false>(ctx, h, g, f, 2, 0, h.n[3], 0, h.n[3] - 1, s))) return rc;
  if ((rc = launch_vlines<true, false>(ctx, h, f, f, 3, -kH, h.n[2] + 2 * kH, -kH + 1, h.n[2] + kH - 2, s)))
    return rc;
  long long blocks = 0;
  if ((rc = launch_advect_4d_fused(ctx, h, f, g, dt, &groups, &blocks, s))) return rc;
  if ((rc = launch_rho_finish(ctx, groups, s))) return rc;
  if ((rc = launch_field_poisson(ctx, s))) return rc;
  if ((rc = launch_diags(ctx, iter, s))) return rc;
  const double scale = h.dx[0] * h.dx[1] * h.dx[2] * h.dx[3];
  k_mpi_l2_finish<<<1, 32, 0, s>>>(ctx->mpi_part, blocks, scale, ctx->l2norm + iter);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

}  // extern "C"
