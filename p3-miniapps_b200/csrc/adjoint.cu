// Reverse mode of the vlp4d step: the discrete adjoint of what vlp4d_step
// computes, with step checkpointing for runs.
//
// Forward step n (timestep.hpp:14-67, as step_impl runs it):
//   a = XY f                       x then y shifts by dt/2 (linear, fixed tables)
//   rho = dvx*dvy * sum_v a ;  E = D rho     (D: the FP64 spectral field solve)
//   b = VXVY(a; E)                 vx then vy shifts by dt*E(x, y)
//   f' = XY b
// Reverse step, given lambda' = dJ/df':
//   lb = XY^T lambda'
//   gE = dJ/dE: gEx = <lb, (dVX/dEx (x) VY) a>, gEy = <lb, (VX (x) dVY/dEy) a>
//        per (x, y), summed over the velocity plane
//   la = VXVY^T lb + dvx*dvy * broadcast(D^T gE)
//   lambda = XY^T la
// Facts used:
// * a line's gather out[i] = sum_k w_k in[(i+m+k) mod n] has as transpose the
//   gather with offset (-m-5) mod n and reversed weights, so XY^T and
//   VXVY^T are the forward kernels (k_plane, k_vslab or the generic ones)
//   run with transposed line tables; x and y sweeps commute exactly (their
//   weights depend on different indices), and so do vx and vy, so the
//   forward kernels' sweep order also serves the transposes;
// * a shift's weights depend on E through the foot position d only:
//   dd/dE = -dt/dh inside a cell, so dw_k/dE = lag_basis5'(d)_k * (-dt/dh);
// * D is linear and translation-invariant (the rho -= 1 of cases 10/20 only
//   touches the zeroed mode), so D^T is the correlation with D's impulse
//   responses hx, hy: (D^T g)^ = conj(hx^) gx^ + conj(hy^) gy^.  The
//   impulse responses are computed once by running the forward field solve
//   on a unit impulse, so the transpose is exact for whatever the forward
//   FFT path does (including its treatment of the Nyquist modes).
//
// Objective of the run-level API: J(f_N) = dx*dy * sum (Ex^2 + Ey^2), the
// electric energy of the field solved from the final state.
#include <cmath>
#include <vector>

#include "internal.cuh"
#include "stencil.cuh"

using vlp4d::StencilTable;

struct vlp4d_adjoint {
  vlp4d_ctx *ctx = nullptr;
  int nsteps = 0, every = 0;
  // every = 0 at creation: the forward sweep keeps the stage input and field
  // of every step (seg, seg_e hold nsteps), the reverse sweep recomputes
  // nothing; `every` is then nsteps and ckpt is empty.
  bool store_all = false;
  size_t fbytes = 0;
  std::vector<void *> ckpt;  // f at steps 0, every, 2*every, ...
  std::vector<void *> seg;   // a = XY f of each step of a segment (every)
  // Ex, Ey of each step of a segment, laid out as the context's fields
  // (Ey fstride after Ex, 2 x fstride per step): one copy saves both.
  double *seg_e = nullptr;
  void *P[2] = {nullptr, nullptr};  // forward work / final state
  void *W[2] = {nullptr, nullptr};  // reverse-step work
  void *L[2] = {nullptr, nullptr};  // adjoint states
  cudaStream_t own = nullptr;       // used when the caller passes the legacy stream
  // CUDA graphs of the forward and reverse sweeps, keyed by the caller's
  // buffers; use_graphs is cleared if a capture fails (eager from then on).
  bool use_graphs = true;
  cudaGraphExec_t g_fwd = nullptr, g_bwd = nullptr;
  const void *k_fwd[2] = {nullptr, nullptr}, *k_bwd = nullptr;
  // FP64 2D work: dJ/dEx, dJ/dEy, dJ/drho, the objective, saved fields.
  double *gex = nullptr, *gey = nullptr, *lam_rho = nullptr, *d_J = nullptr, *save = nullptr;
  double *gpart = nullptr;  // per-segment partial sums of gE
  int gsegs = 0;
  cufftDoubleComplex *hx_hat = nullptr, *hy_hat = nullptr;  // spectra of the impulse responses
  // Forward transforms of gex and gey (adjacent, n2 apart) into the
  // context's ex_hat and ey_hat as one batched plan.
  cufftHandle plan_g2 = 0;
  bool have_plan_g2 = false;
  bool field_linear = true;  // false for the analytic-field cases 2 and 6
  StencilTable tab_x_adj, tab_y_adj, tab_vx_adj, tab_vy_adj;
  // The transposed x/y half step applied twice as 11-tap lines: the last
  // x/y pass of one reverse step and the first of the step before it in one
  // k_plane_xyxy pass (valid = false: two x/y passes instead).
  StencilTable tab_x11_adj, tab_y11_adj;
  double *dw_vx = nullptr, *dw_vy = nullptr;  // dw/dE per v line (6 each, FP64)
  bool have_forward = false;
  double J = 0.0;
};

namespace vlp4d {
namespace {

// The v tables of one direction of a reverse step, from E: the forward
// stencils (into the context's tables), the transposed ones and the weight
// derivatives, from one line_stencil per line.  grid.y selects the
// direction (vx, vy): one launch for all six tables.
struct VtableAdjJob {
  const double *e;
  double hmin, hmax;
  int n;
  StencilTable fwd, adj;  // span / span_C set: also the chunk spans (the vy direction)
  double *dw;
};
__global__ void k_build_vtables_rev(VtableAdjJob jx, VtableAdjJob jy, int lines, double dt) {
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  const bool on = line < lines;
  const VtableAdjJob &j = blockIdx.y ? jy : jx;
  int ms = 0, mt = 0;
  if (on) {
    const LineStencil s = line_stencil(__dmul_rn(dt, j.e[line]), j.hmin, j.hmax, j.n);
    const LineStencil t = adjoint_stencil(s, j.n);
    float f[6], fa[6];
    weights_to_f32(s.w, f);
    weights_to_f32(t.w, fa);
    j.fwd.m[line] = s.m;
    j.adj.m[line] = t.m;
    ms = s.m;
    mt = t.m;
    double dc[6];
    lag_basis5_deriv(s.d, dc);
    const double scale = -dt / ((j.hmax - j.hmin) / (double)j.n);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      j.fwd.w[6 * line + k] = s.w[k];
      j.fwd.wf[6 * line + k] = f[k];
      j.adj.w[6 * line + k] = t.w[k];
      j.adj.wf[6 * line + k] = fa[k];
      j.dw[6 * line + k] = dc[k] * scale;
    }
  }
  if (j.fwd.span_C) chunk_span(on, signed_offset(ms, j.n), line, j.fwd.span_C, j.fwd.span);
  if (j.adj.span_C) chunk_span(on, signed_offset(mt, j.n), line, j.adj.span_C, j.adj.span);
}

// gE partial sums.  Block (32 columns) x (GY vx groups); grid (column
// chunks, vy segments).  A thread owns one column ixy and the output vx rows
// ty, ty+GY, ...; for each it streams the input vy rows of its segment (the
// Q outputs plus the five-row halo, starting at the column's vy offset),
// keeping the last six vx-swept rows (value A and vx-derivative B) in a
// ring, and accumulates lb * (sum_l wy_l B_l) and lb * (sum_l dwy_l A_l).
// The ring slot of row r is r mod 6, static after unrolling by six.
template <typename T>
__global__ void __launch_bounds__(256) k_vgrad(const T *__restrict__ a, const T *__restrict__ lb, int nxy, int nvx,
                                               int nvy, int Q, StencilTable tvx, StencilTable tvy,
                                               const double *__restrict__ dwx, const double *__restrict__ dwy,
                                               double *__restrict__ part) {
  const int tx = threadIdx.x, ty = threadIdx.y, GY = blockDim.y;
  const int ixy = blockIdx.x * 32 + tx;
  const int seg = blockIdx.y;
  const int ivy0 = seg * Q;
  const int q = min(Q, nvy - ivy0);
  double gx = 0., gy = 0.;
  if (ixy < nxy && q > 0) {
    const long long vstride = nxy, ystride = (long long)nxy * nvx;
    double wx[6], dx[6], wy[6], dy[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      wx[k] = tvx.w[6 * (long long)ixy + k];
      dx[k] = dwx[6 * (long long)ixy + k];
      wy[k] = tvy.w[6 * (long long)ixy + k];
      dy[k] = dwy[6 * (long long)ixy + k];
    }
    const int mx = tvx.m[ixy], my = tvy.m[ixy];
    for (int ivx = ty; ivx < nvx; ivx += GY) {
      long long toff[6];
      int j = ivx + mx;
      if (j >= nvx) j -= nvx;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        toff[k] = (long long)j * vstride + ixy;
        if (++j == nvx) j = 0;
      }
      double A[6], B[6];
      int row = (ivy0 + my) % nvy;
      const int nrows = q + 5;
      for (int r0 = 0; r0 < nrows; r0 += 6) {
#pragma unroll
        for (int u = 0; u < 6; ++u) {
          const int r = r0 + u;
          if (r >= nrows) break;
          const T *p = a + (long long)row * ystride;
          double s = 0., sd = 0.;
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            const double v = (double)__ldg(p + toff[k]);
            s = fma(wx[k], v, s);
            sd = fma(dx[k], v, sd);
          }
          A[u] = s;
          B[u] = sd;
          if (++row == nvy) row = 0;
          if (r >= 5) {
            const int ivy = ivy0 + r - 5;
            const double l = (double)__ldg(lb + (long long)ivy * ystride + (long long)ivx * vstride + ixy);
            double sx = 0., sy = 0.;
#pragma unroll
            for (int t = 0; t < 6; ++t) {
              sx = fma(wy[t], B[(u + 1 + t) % 6], sx);
              sy = fma(dy[t], A[(u + 1 + t) % 6], sy);
            }
            gx = fma(l, sx, gx);
            gy = fma(l, sy, gy);
          }
        }
      }
    }
  }
  // Sum the vx groups in a fixed order.
  __shared__ double sx[8][32], sy[8][32];
  sx[ty][tx] = gx;
  sy[ty][tx] = gy;
  __syncthreads();
  if (ty == 0 && ixy < nxy) {
    double ax = 0., ay = 0.;
    for (int g = 0; g < GY; ++g) {
      ax += sx[g][tx];
      ay += sy[g][tx];
    }
    part[(2LL * seg) * nxy + ixy] = ax;
    part[(2LL * seg + 1) * nxy + ixy] = ay;
  }
}

// Asynchronous 4- or 8-byte global-to-shared copies (through L1), in
// commit groups per thread.
template <int BYTES>
__device__ __forceinline__ void cp_async_small(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (BYTES == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_groups() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Element pairs of k_vgrad_v: two independent sums advanced by one packed
// instruction in FP32 (fma.rn.f32x2 / mul.rn.f32x2: per-lane results equal
// to the scalar fmaf / multiply), component-wise in FP64.
template <typename T>
struct VgPair;
template <>
struct VgPair<float> {
  using P = float2;
  static __device__ __forceinline__ P mk(float a, float b) { return make_float2(a, b); }
  static __device__ __forceinline__ P mul(P a, P b) { return __fmul2_rn(a, b); }
  static __device__ __forceinline__ P fma2(P a, P b, P c) { return __ffma2_rn(a, b, c); }
};
template <>
struct VgPair<double> {
  using P = double2;
  static __device__ __forceinline__ P mk(double a, double b) { return make_double2(a, b); }
  static __device__ __forceinline__ P mul(P a, P b) { return make_double2(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)); }
  static __device__ __forceinline__ P fma2(P a, P b, P c) { return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y)); }
};

// The same sums with the vx taps shared: thread (cw, g) of a block owns
// column ixy = blockIdx.x*CW + cw and the V consecutive output vx rows
// g*V .. g*V+V-1 (blockDim = CW x nvx/V), so one input row costs V+5 loads
// for V outputs.  The stencil sums and the row's products with lb run in
// the element type, the accumulation over rows in FP64.  Register ring of
// the vx-swept rows: slot r mod 6, static after unrolling by six.
//
// Loads: each thread copies its own V+5 taps and V adjoint values of a row
// into its private slots of a shared-memory ring of S rows with cp.async,
// S-1 rows ahead of the row it computes (one commit group per row; the
// slot written is the one read a row earlier, so no copy lands in a slot
// still being read).  Slots are laid out [slot][element][thread]: a warp's
// accesses are consecutive words.  Nothing is shared between threads
// until the final reduction.
template <typename T, int V, int S>
__global__ void __launch_bounds__(512) k_vgrad_v(const T *__restrict__ a, const T *__restrict__ lb, int nxy,
                                                 int nvx, int nvy, int Q, StencilTable tvx, StencilTable tvy,
                                                 const double *__restrict__ dwx, const double *__restrict__ dwy,
                                                 double *__restrict__ part) {
  static_assert(S >= 2, "at least one row in flight");
  constexpr int NE = V + 5 + V;  // elements of one row per thread
  constexpr int D = S - 1;       // rows in flight ahead of the computed one
  extern __shared__ __align__(16) unsigned char vg_smem[];
  const int CW = blockDim.x;
  const int G = blockDim.y;
  const int cw = threadIdx.x, g = threadIdx.y;
  const int nth = CW * G, tid = g * CW + cw;
  T *ring = reinterpret_cast<T *>(vg_smem);                               // [S][nth][NE]
  double *red = reinterpret_cast<double *>(vg_smem + sizeof(T) * S * NE * nth);  // [2][G][CW]
  const int ixy = blockIdx.x * CW + cw;
  const int seg = blockIdx.y;
  const int ivy0 = seg * Q;
  const int q = min(Q, nvy - ivy0);
  const int vx0 = g * V;
  double gx = 0., gy = 0.;
  if (ixy < nxy && q > 0) {
    const long long vstride = nxy, ystride = (long long)nxy * nvx;
    // Stencil sums in the element type (FP32 sums of FP32 data are
    // accurate to ~1e-7 for a gradient); products with lb and the
    // accumulation in FP64.
    // Weight pairs: (dwx, wx) for the vx sums (B, A) of a row, (wy, dwy) for
    // the vy sums (sx, sy) = (sum wy B, sum dwy A).
    using VP = VgPair<T>;
    using P = typename VP::P;
    P wdx[6], wdy[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      wdx[k] = VP::mk((T)dwx[6 * (long long)ixy + k], (T)tvx.w[6 * (long long)ixy + k]);
      wdy[k] = VP::mk((T)tvy.w[6 * (long long)ixy + k], (T)dwy[6 * (long long)ixy + k]);
    }
    // Element offsets within a vy row of this thread's vx tap rows
    // (nvx * nxy < 2^31) and of its lb rows.
    int toff[V + 5];
    {
      int j = vx0 + tvx.m[ixy];
      if (j >= nvx) j -= nvx;
#pragma unroll
      for (int k = 0; k < V + 5; ++k) {
        toff[k] = j * nxy;
        if (++j == nvx) j = 0;
      }
    }
    const int my = tvy.m[ixy];
    P BA[6][V];  // ring of the vx-swept rows: (B, A) = (sum dwx t, sum wx t)
    const int nrows = q + 5;
    // Running pointers: the a row of the next row to load (periodic in vy),
    // the lb row it brings (from row 5 on), the ring slots of the next row
    // to load and to compute.  The ring is [slot][thread][element]: element
    // offsets are immediates, and the odd (FP32) or 18-word (FP64) thread
    // stride keeps a warp's accesses on distinct banks.
    int lrow = (ivy0 + my) % nvy;
    const T *arow = a + (long long)lrow * ystride + ixy;
    const T *lnext = lb + (long long)ivy0 * ystride + (long long)vx0 * vstride + ixy;
    T *const ring0 = ring + (size_t)tid * NE;
    const size_t slot_elems = (size_t)nth * NE;
    T *wptr = ring0;
    const T *rptr = ring0;
    // Row rr of the segment into the next slot (an empty group past the
    // last row, so that every row has one commit group).
    auto issue = [&](int rr) {
      if (rr < nrows) {
#pragma unroll
        for (int k = 0; k < V + 5; ++k) cp_async_small<sizeof(T)>(wptr + k, arow + toff[k]);
        if (rr >= 5) {
#pragma unroll
          for (int i = 0; i < V; ++i) cp_async_small<sizeof(T)>(wptr + V + 5 + i, lnext + i * nxy);
          lnext += ystride;
        }
        if (++lrow == nvy) {
          lrow = 0;
          arow = a + ixy;
        } else {
          arow += ystride;
        }
      }
      wptr = wptr + slot_elems == ring0 + S * slot_elems ? ring0 : wptr + slot_elems;
      cp_async_commit_group();
    };
#pragma unroll
    for (int rr = 0; rr < D; ++rr) issue(rr);
    for (int r0 = 0; r0 < nrows; r0 += 6) {
#pragma unroll
      for (int u = 0; u < 6; ++u) {
        const int r = r0 + u;
        if (r >= nrows) break;
        // Rows up to r have landed (D groups committed after row r's).
        cp_async_wait_groups<D - 1>();
        issue(r + D);  // into slot (r + D) mod S = (r - 1) mod S, read a row ago
        const T *src = rptr;
        rptr = rptr + slot_elems == ring0 + S * slot_elems ? ring0 : rptr + slot_elems;
        T t[V + 5];
#pragma unroll
        for (int k = 0; k < V + 5; ++k) t[k] = src[k];
#pragma unroll
        for (int i = 0; i < V; ++i) {
          P ba = VP::mul(wdx[0], VP::mk(t[i], t[i]));
#pragma unroll
          for (int k = 1; k < 6; ++k) ba = VP::fma2(wdx[k], VP::mk(t[i + k], t[i + k]), ba);
          BA[u][i] = ba;
        }
        if (r >= 5) {
          // The row's V products with lb summed in the element type, then
          // added to the FP64 sums (two conversions per row, not 3V).
          P pxy = VP::mk(0, 0);
#pragma unroll
          for (int i = 0; i < V; ++i) {
            const T l = src[V + 5 + i];
            P sxy = VP::mul(wdy[0], BA[(u + 1) % 6][i]);
#pragma unroll
            for (int k = 1; k < 6; ++k) sxy = VP::fma2(wdy[k], BA[(u + 1 + k) % 6][i], sxy);
            pxy = VP::fma2(VP::mk(l, l), sxy, pxy);
          }
          gx += (double)pxy.x;
          gy += (double)pxy.y;
        }
      }
    }
    cp_async_wait_groups<0>();
  }
  // Sum the vx groups of each column in a fixed order.
  red[g * CW + cw] = gx;
  red[(G + g) * CW + cw] = gy;
  __syncthreads();
  if (g == 0 && ixy < nxy) {
    double ax = 0., ay = 0.;
    for (int k = 0; k < G; ++k) {
      ax += red[k * CW + cw];
      ay += red[(G + k) * CW + cw];
    }
    part[(2LL * seg) * nxy + ixy] = ax;
    part[(2LL * seg + 1) * nxy + ixy] = ay;
  }
}

// Ring rows of k_vgrad_v: two rows in flight (three to five rows measured
// no faster; V = 2 with five rows in flight slower, 72.8 against 63.1 us at
// 64^4), and its shared memory.
template <typename T, int V>
constexpr int vgrad_slots() {
  return 3;
}
template <typename T, int V>
size_t vgrad_smem(int nth, int gy, int cw) {
  return sizeof(T) * vgrad_slots<T, V>() * (2 * V + 5) * (size_t)nth + sizeof(double) * 2 * gy * cw;
}

__global__ void k_vgrad_finish(const double *__restrict__ part, int nseg, int nxy, double *__restrict__ gex,
                               double *__restrict__ gey) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nxy) return;
  double ax = 0., ay = 0.;
  for (int s = 0; s < nseg; ++s) {
    ax += part[(2LL * s) * nxy + i];
    ay += part[(2LL * s + 1) * nxy + i];
  }
  gex[i] = ax;
  gey[i] = ay;
}

// lam_hat = (conj(hx_hat) gx_hat + conj(hy_hat) gy_hat) / (nx*ny).
__global__ void k_field_transpose(const cufftDoubleComplex *__restrict__ gx, const cufftDoubleComplex *__restrict__ gy,
                                  const cufftDoubleComplex *__restrict__ hx, const cufftDoubleComplex *__restrict__ hy,
                                  cufftDoubleComplex *__restrict__ out, int nh, double norm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nh) return;
  const cufftDoubleComplex a = gx[i], b = gy[i], p = hx[i], q = hy[i];
  cufftDoubleComplex r;
  r.x = (p.x * a.x + p.y * a.y + q.x * b.x + q.y * b.y) * norm;
  r.y = (p.x * a.y - p.y * a.x + q.x * b.y - q.y * b.x) * norm;
  out[i] = r;
}

// f[v*nxy + ixy] (+)= scale * col[ixy] for every velocity cell v.
template <typename T, bool ADD>
__global__ void k_columns(T *__restrict__ f, const double *__restrict__ col, double scale, long long nxy,
                          long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const double c = scale * col[i % nxy];
    f[i] = ADD ? (T)((double)f[i] + c) : (T)c;
  }
}

// J = dxdy * sum (ex^2 + ey^2) (Kahan, one block, fixed order) and
// gex = 2 dxdy ex, gey = 2 dxdy ey.
__global__ void k_energy(const double *__restrict__ ex, const double *__restrict__ ey, long long n, double dxdy,
                         double *__restrict__ J, double *__restrict__ gex, double *__restrict__ gey) {
  double s = 0., c = 0.;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    const double a = ex[i], b = ey[i];
    const double y = (a * a + b * b) - c;
    const double t = s + y;
    c = (t - s) - y;
    s = t;
    gex[i] = 2. * dxdy * a;
    gey[i] = 2. * dxdy * b;
  }
  s -= c;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double ws[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) ws[warp] = s;
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    s = lane < nw ? ws[lane] : 0.;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) *J = s * dxdy;
  }
}

int grid_cap(long long total, int threads, int sms) {
  long long b = (total + threads - 1) / threads;
  const long long cap = (long long)sms * 16;
  return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

}  // namespace
}  // namespace vlp4d

namespace vlp4d {
namespace {

// Transposed x (dim 0) and y (dim 1) tables for shifts by dt*v, built on the
// host like ensure_xy_table's and uploaded.
int build_xy_adj(vlp4d_ctx *c, int dim, double dt, StencilTable &t, cudaStream_t s) {
  const int vdim = dim == 0 ? 2 : 3;
  const int lines = c->g.n[vdim];
  int rc = alloc_table(t, lines);
  if (rc) return rc;
  std::vector<int> hm(lines);
  std::vector<double> hw(6 * (size_t)lines);
  std::vector<float> hwf(6 * (size_t)lines);
  for (int l = 0; l < lines; ++l) {
    const double v = c->g.minp[vdim] + l * c->g.dx[vdim];
    const LineStencil st = adjoint_stencil(line_stencil(dt * v, c->g.minp[dim], c->g.maxp[dim], c->g.n[dim]), c->g.n[dim]);
    hm[l] = st.m;
    float f[6];
    weights_to_f32(st.w, f);
    for (int k = 0; k < 6; ++k) {
      hw[6 * l + k] = st.w[k];
      hwf[6 * l + k] = f[k];
    }
  }
  VLP4D_CUDA_TRY(cudaMemcpyAsync(t.m, hm.data(), sizeof(int) * lines, cudaMemcpyHostToDevice, s));
  VLP4D_CUDA_TRY(cudaMemcpyAsync(t.w, hw.data(), sizeof(double) * 6 * lines, cudaMemcpyHostToDevice, s));
  VLP4D_CUDA_TRY(cudaMemcpyAsync(t.wf, hwf.data(), sizeof(float) * 6 * lines, cudaMemcpyHostToDevice, s));
  VLP4D_CUDA_TRY(cudaStreamSynchronize(s));
  t.dt = dt;
  t.valid = true;
  return VLP4D_OK;
}

// Spectra of the field solve's impulse responses (section comment above).
// The context's rho/Ex/Ey are saved and restored around the probe solve.
int field_transpose_setup(vlp4d_adjoint *A, cudaStream_t s) {
  vlp4d_ctx *c = A->ctx;
  const long long n2 = c->g.nxy();
  if (c->dom.idcase == 2 || c->dom.idcase == 6) {
    A->field_linear = false;
    return VLP4D_OK;
  }
  {
    int n[2] = {c->g.n[1], c->g.n[0]};
    int inembed[2] = {c->g.n[1], c->g.n[0]}, onembed[2] = {c->g.n[1], c->g.n[0] / 2 + 1};
    if (cufftPlanMany(&A->plan_g2, 2, n, inembed, 1, (int)n2, onembed, 1, (int)c->hstride, CUFFT_D2Z, 2) !=
        CUFFT_SUCCESS)
      return fail_msg(VLP4D_ERR_CUDA, "adjoint: cufftPlanMany D2Z (batch 2) failed");
    A->have_plan_g2 = true;
  }
  VLP4D_CUDA_TRY(cudaMemcpyAsync(A->save, c->rho, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
  VLP4D_CUDA_TRY(cudaMemcpyAsync(A->save + n2, c->ex, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
  VLP4D_CUDA_TRY(cudaMemcpyAsync(A->save + 2 * n2, c->ey, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
  static const double one = 1.0;
  VLP4D_CUDA_TRY(cudaMemsetAsync(c->rho, 0, sizeof(double) * n2, s));
  VLP4D_CUDA_TRY(cudaMemcpyAsync(c->rho, &one, sizeof(double), cudaMemcpyHostToDevice, s));
  int rc = launch_field_poisson(c, s);
  if (rc) return rc;
  VLP4D_CUFFT_TRY(cufftSetStream(c->plan_fwd, s));
  VLP4D_CUFFT_TRY(cufftExecD2Z(c->plan_fwd, c->ex, A->hx_hat));
  VLP4D_CUFFT_TRY(cufftExecD2Z(c->plan_fwd, c->ey, A->hy_hat));
  VLP4D_CUDA_TRY(cudaMemcpyAsync(c->rho, A->save, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
  VLP4D_CUDA_TRY(cudaMemcpyAsync(c->ex, A->save + n2, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
  VLP4D_CUDA_TRY(cudaMemcpyAsync(c->ey, A->save + 2 * n2, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
  VLP4D_CUDA_TRY(cudaStreamSynchronize(s));
  return VLP4D_OK;
}

// lam_rho = D^T (gex, gey).
int field_transpose(vlp4d_adjoint *A, cudaStream_t s) {
  vlp4d_ctx *c = A->ctx;
  const int nx = c->g.n[0], ny = c->g.n[1];
  if (!A->field_linear) {
    VLP4D_CUDA_TRY(cudaMemsetAsync(A->lam_rho, 0, sizeof(double) * c->g.nxy(), s));
    return VLP4D_OK;
  }
  if (field_cluster_t_available(c))
    return launch_field_transpose_cluster(c, A->gex, A->gey, A->hx_hat, A->hy_hat, A->lam_rho, s);
  VLP4D_CUFFT_TRY(cufftSetStream(A->plan_g2, s));
  VLP4D_CUFFT_TRY(cufftSetStream(c->plan_bwd, s));
  VLP4D_CUFFT_TRY(cufftExecD2Z(A->plan_g2, A->gex, c->ex_hat));  // gex, gey -> ex_hat, ey_hat
  const int nh = (nx / 2 + 1) * ny;
  k_field_transpose<<<(nh + 255) / 256, 256, 0, s>>>(c->ex_hat, c->ey_hat, A->hx_hat, A->hy_hat, c->rho_hat, nh,
                                                     1.0 / ((double)nx * ny));
  VLP4D_LAUNCH_CHECK();
  VLP4D_CUFFT_TRY(cufftExecZ2D(c->plan_bwd, c->rho_hat, A->lam_rho));
  return VLP4D_OK;
}

// gE from the stage input a (of the vx/vy pass) and lb (the adjoint after it).
int launch_vgrad(vlp4d_adjoint *A, const void *a, const void *lb, cudaStream_t s) {
  vlp4d_ctx *c = A->ctx;
  const int nxy = (int)c->g.nxy(), nvx = c->g.n[2], nvy = c->g.n[3];
  const int bx = (nxy + 31) / 32;
  int nseg = (2 * c->num_sms + bx - 1) / bx;
  if (nseg < 1) nseg = 1;
  if (nseg > nvy) nseg = nvy;
  if (nseg > A->gsegs) nseg = A->gsegs;
  const int Q = (nvy + nseg - 1) / nseg;
  nseg = (nvy + Q - 1) / Q;
  // Shared-tap kernel: V vx rows per thread (4 in FP32, 2 in FP64), nvx/V
  // threads per column, as many columns per block as fit 512 threads.
  const int V = c->dtype == VLP4D_F32 ? 4 : 2;
  if (nvx % V == 0 && nvx / V <= 512) {
    const int gy = nvx / V;
    int cw = 512 / gy;
    if (cw > 32) cw = 32;
    if (getenv("VLP4D_VGRAD_CW")) {  // columns per block, for tuning sweeps
      const int f = atoi(getenv("VLP4D_VGRAD_CW"));
      if (f >= 1 && f <= cw) cw = f;
    }
    const int bxv = (nxy + cw - 1) / cw;
    // vy segments: a block streams Qv + 5 rows of its segment, one block per
    // SM at a time, so the pass takes about ceil(blocks / SMs) * (Qv + 5)
    // row times; the segment count minimises that, one wave on part of the
    // SMs included (64^4 FP32: 128 blocks of one segment, 69 row times,
    // measured 2-3 us faster than 256 blocks of two, 2 x 37; VLP4D_VGRAD_SEGS
    // overrides).
    int ns = 0;
    {
      long long best = -1;
      const int forced = getenv("VLP4D_VGRAD_SEGS") ? atoi(getenv("VLP4D_VGRAD_SEGS")) : 0;
      for (int k = 1; k <= nvy && k <= A->gsegs; ++k) {
        const int q = (nvy + k - 1) / k;
        if ((nvy + q - 1) / q != k) continue;  // the same segments as a smaller count
        const long long blocks = (long long)bxv * k;
        if (forced && k != forced) continue;
        const long long cost = (blocks + c->num_sms - 1) / c->num_sms * (q + 5);
        if (best < 0 || cost < best) {
          best = cost;
          ns = k;
        }
      }
      if (!ns) ns = 1;
    }
    const int Qv = (nvy + ns - 1) / ns;
    ns = (nvy + Qv - 1) / Qv;
    dim3 gridv(bxv, ns), blockv(cw, gy);
    // One segment: its partials are gex, gey themselves (gey follows gex
    // as the partials of a segment follow each other).
    double *part = ns == 1 ? A->gex : A->gpart;
    if (c->dtype == VLP4D_F64) {
      auto kern = k_vgrad_v<double, 2, vgrad_slots<double, 2>()>;
      const size_t sm = vgrad_smem<double, 2>(cw * gy, gy, cw);
      VLP4D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      kern<<<gridv, blockv, sm, s>>>((const double *)a, (const double *)lb, nxy, nvx, nvy, Qv, c->tab_vx, c->tab_vy,
                                     A->dw_vx, A->dw_vy, part);
    } else {
      auto kern = k_vgrad_v<float, 4, vgrad_slots<float, 4>()>;
      const size_t sm = vgrad_smem<float, 4>(cw * gy, gy, cw);
      VLP4D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      kern<<<gridv, blockv, sm, s>>>((const float *)a, (const float *)lb, nxy, nvx, nvy, Qv, c->tab_vx, c->tab_vy,
                                     A->dw_vx, A->dw_vy, part);
    }
    VLP4D_LAUNCH_CHECK();
    if (ns > 1) {
      k_vgrad_finish<<<(nxy + 255) / 256, 256, 0, s>>>(A->gpart, ns, nxy, A->gex, A->gey);
      VLP4D_LAUNCH_CHECK();
    }
    return VLP4D_OK;
  }
  dim3 grid(bx, nseg), block(32, 8);
  if (c->dtype == VLP4D_F64)
    k_vgrad<double><<<grid, block, 0, s>>>((const double *)a, (const double *)lb, nxy, nvx, nvy, Q, c->tab_vx,
                                           c->tab_vy, A->dw_vx, A->dw_vy, A->gpart);
  else
    k_vgrad<float><<<grid, block, 0, s>>>((const float *)a, (const float *)lb, nxy, nvx, nvy, Q, c->tab_vx,
                                          c->tab_vy, A->dw_vx, A->dw_vy, A->gpart);
  VLP4D_LAUNCH_CHECK();
  k_vgrad_finish<<<(nxy + 255) / 256, 256, 0, s>>>(A->gpart, nseg, nxy, A->gex, A->gey);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

int launch_columns(vlp4d_adjoint *A, void *f, bool add, double scale, cudaStream_t s) {
  vlp4d_ctx *c = A->ctx;
  const long long nxy = c->g.nxy(), total = c->g.cells();
  const int threads = 256, blocks = grid_cap(total, threads, c->num_sms);
  if (c->dtype == VLP4D_F64) {
    if (add) k_columns<double, true><<<blocks, threads, 0, s>>>((double *)f, A->lam_rho, scale, nxy, total);
    else k_columns<double, false><<<blocks, threads, 0, s>>>((double *)f, A->lam_rho, scale, nxy, total);
  } else {
    if (add) k_columns<float, true><<<blocks, threads, 0, s>>>((float *)f, A->lam_rho, scale, nxy, total);
    else k_columns<float, false><<<blocks, threads, 0, s>>>((float *)f, A->lam_rho, scale, nxy, total);
  }
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

// J of the field solved from f into A->d_J, lam = dJ/df.
int energy_grad(vlp4d_adjoint *A, const void *f, void *lam, cudaStream_t s) {
  vlp4d_ctx *c = A->ctx;
  int rc;
  if ((rc = launch_field_rho(c, f, s))) return rc;
  if ((rc = launch_field_poisson(c, s))) return rc;
  k_energy<<<1, 1024, 0, s>>>(c->ex, c->ey, c->g.nxy(), c->g.dx[0] * c->g.dx[1], A->d_J, A->gex, A->gey);
  VLP4D_LAUNCH_CHECK();
  if ((rc = field_transpose(A, s))) return rc;
  return launch_columns(A, lam, false, c->g.dx[2] * c->g.dx[3], s);
}

// The middle of a reverse step, from lb = XY^T lam_next (in lb) to
// la = VXVY^T lb + dvx dvy broadcast(dJ/drho) (into la): the v tables and
// their E-derivatives from the stored field e of the step (NULL: the
// context's Ex, Ey), dJ/dE from the stored stage input a, dJ/drho.
int reverse_core(vlp4d_adjoint *A, const void *a, const double *e, const void *lb, void *la, cudaStream_t s) {
  vlp4d_ctx *c = A->ctx;
  const double dt = c->dom.dt;
  const long long n2 = c->g.nxy();
  const int lines = (int)n2;
  int rc;
  // The step's field: stored (Ey fstride after Ex) or the context's own.
  const double *ex = e ? e : c->ex, *ey = e ? e + c->fstride : c->ey;
  if ((rc = alloc_table(c->tab_vx, lines)) || (rc = alloc_table(c->tab_vy, lines))) return rc;
  // The vy chunk spans of the v-slab pass (forward and transposed tables)
  // where it runs on this shape.
  const int C = vslab_chunk_cols(c);
  c->tab_vy.span_C = A->tab_vy_adj.span_C = 0;
  if (C && alloc_span(c->tab_vy, C) == VLP4D_OK && alloc_span(A->tab_vy_adj, C) == VLP4D_OK)
    c->tab_vy.span_C = A->tab_vy_adj.span_C = C;
  c->tab_vx.span_C = A->tab_vx_adj.span_C = 0;
  const int threads = 256, blocks = (lines + threads - 1) / threads;
  const VtableAdjJob jx = {ex, c->g.minp[2], c->g.maxp[2], c->g.n[2], c->tab_vx, A->tab_vx_adj, A->dw_vx};
  const VtableAdjJob jy = {ey, c->g.minp[3], c->g.maxp[3], c->g.n[3], c->tab_vy, A->tab_vy_adj, A->dw_vy};
  k_build_vtables_rev<<<dim3((unsigned)blocks, 2u), threads, 0, s>>>(jx, jy, lines, dt);
  VLP4D_LAUNCH_CHECK();
  c->tab_vx.valid = c->tab_vy.valid = true;
  // dJ/dE, then dJ/drho.
  if ((rc = launch_vgrad(A, a, lb, s))) return rc;
  if ((rc = field_transpose(A, s))) return rc;
  // la = VXVY^T lb + dvx dvy broadcast(dJ/drho), the broadcast folded into
  // the v-slab pass where it runs.
  const double scale = c->g.dx[2] * c->g.dx[3];
  rc = launch_advect_vxvy_tables(c, lb, la, &A->tab_vx_adj, &A->tab_vy_adj, s, A->lam_rho, scale);
  if (rc == VLP4D_ERR_UNSUPPORTED) {
    if ((rc = advect_vxvy_any(c, lb, la, &A->tab_vx_adj, &A->tab_vy_adj, s))) return rc;
    if ((rc = launch_columns(A, la, true, scale, s))) return rc;
  } else if (rc) {
    return rc;
  }
  return VLP4D_OK;
}

// The reverse step from the stored stage input a (= XY f) and its field E:
// lam_out = (d step/d f)^T lam_next = XY^T (reverse_core(XY^T lam_next)).
int step_adjoint_stored(vlp4d_adjoint *A, const void *a, const double *e, const void *lam_next, void *lam_out,
                        cudaStream_t s) {
  vlp4d_ctx *c = A->ctx;
  int rc;
  if ((rc = advect_xy_any(c, lam_next, A->W[1], &A->tab_x_adj, &A->tab_y_adj, s))) return rc;
  if ((rc = reverse_core(A, a, e, A->W[1], A->W[0], s))) return rc;
  return advect_xy_any(c, A->W[0], lam_out, &A->tab_x_adj, &A->tab_y_adj, s);
}

// The reverse step at the state f_state: recompute a = XY f and its field.
int step_adjoint(vlp4d_adjoint *A, const void *f_state, const void *lam_next, void *lam_out, cudaStream_t s) {
  vlp4d_ctx *c = A->ctx;
  int rc;
  if ((rc = advect_xy_moment(c, f_state, A->P[0], 0.5 * c->dom.dt, s))) return rc;
  if ((rc = launch_field_poisson(c, s))) return rc;
  return step_adjoint_stored(A, A->P[0], nullptr, lam_next, lam_out, s);
}

// Ex and Ey of step j of the segment: one copy (Ey sits fstride after Ex in
// both places).
void save_field(vlp4d_adjoint *A, int j, cudaStream_t s) {
  vlp4d_ctx *c = A->ctx;
  const long long n2 = c->g.nxy();
  double *e = A->seg_e + 2 * (long long)c->fstride * j;
  cudaMemcpyAsync(e, c->ex, sizeof(double) * ((long long)c->fstride + n2), cudaMemcpyDeviceToDevice, s);
}

// The closing x/y half step of one step and the opening one (with the
// moment) of the next: one k_plane_xyxy pass where it is the faster kernel,
// else two x/y passes through `tmp`.
int xy_xy_moment(vlp4d_ctx *c, const void *in, void *out, void *tmp, cudaStream_t s) {
  StencilTable *tx = nullptr, *ty = nullptr;
  int rc;
  if ((rc = ensure_xy_table(c, 0, 0.5 * c->dom.dt, &tx, s))) return rc;
  if ((rc = ensure_xy_table(c, 1, 0.5 * c->dom.dt, &ty, s))) return rc;
  if (xyxy_join(c)) {
    rc = launch_advect_xyxy(c, in, out, tx, ty, s);
    if (rc != VLP4D_ERR_UNSUPPORTED) return rc;
  }
  if ((rc = advect_xy_any(c, in, tmp, tx, ty, s))) return rc;
  return advect_xy_moment(c, tmp, out, 0.5 * c->dom.dt, s);
}

// The stage inputs a = XY f (into seg[0 .. len-1]) and fields E (seg_e) of
// len steps from the state f: the moment pass, then per further step the
// v pass and the joined x/y/x/y pass with the moment; the last step's v pass
// is left to the caller.
int store_segment(vlp4d_adjoint *A, const void *f, int len, cudaStream_t s) {
  vlp4d_ctx *c = A->ctx;
  const double dt = c->dom.dt;
  int rc;
  if ((rc = advect_xy_moment(c, f, A->seg[0], 0.5 * dt, s))) return rc;
  if ((rc = launch_field_poisson(c, s))) return rc;
  save_field(A, 0, s);
  for (int j = 1; j < len; ++j) {
    if ((rc = build_v_tables(c, dt, true, true, s))) return rc;
    if ((rc = advect_vxvy_any(c, A->seg[j - 1], A->W[0], &c->tab_vx, &c->tab_vy, s))) return rc;
    if ((rc = xy_xy_moment(c, A->W[0], A->seg[j], A->W[1], s))) return rc;
    if ((rc = launch_field_poisson(c, s))) return rc;
    save_field(A, j, s);
  }
  return VLP4D_OK;
}

// Forward sweep: nsteps steps from f0, each segment's final state written to
// the next checkpoint (the last one to P[1]); J and dJ/df_N into d_J, L[0].
int forward_body(vlp4d_adjoint *A, const void *f0, void *f_out, cudaStream_t s) {
  vlp4d_ctx *c = A->ctx;
  const double dt = c->dom.dt;
  int rc;
  if (A->store_all) {
    if ((rc = store_segment(A, f0, A->nsteps, s))) return rc;
    // The last step's v pass and closing x/y half step.
    if ((rc = build_v_tables(c, dt, true, true, s))) return rc;
    if ((rc = advect_vxvy_any(c, A->seg[A->nsteps - 1], A->W[0], &c->tab_vx, &c->tab_vy, s))) return rc;
    StencilTable *tx = nullptr, *ty = nullptr;
    if ((rc = ensure_xy_table(c, 0, 0.5 * dt, &tx, s))) return rc;
    if ((rc = ensure_xy_table(c, 1, 0.5 * dt, &ty, s))) return rc;
    if ((rc = advect_xy_any(c, A->W[0], A->P[1], tx, ty, s))) return rc;
    if ((rc = energy_grad(A, A->P[1], A->L[0], s))) return rc;
    if (f_out) VLP4D_CUDA_TRY(cudaMemcpyAsync(f_out, A->P[1], A->fbytes, cudaMemcpyDeviceToDevice, s));
    return VLP4D_OK;
  }
  VLP4D_CUDA_TRY(cudaMemcpyAsync(A->ckpt[0], f0, A->fbytes, cudaMemcpyDeviceToDevice, s));
  const int nseg = (int)A->ckpt.size();
  for (int sg = 0; sg < nseg; ++sg) {
    const int len = A->nsteps - sg * A->every < A->every ? A->nsteps - sg * A->every : A->every;
    void *out = sg + 1 < nseg ? A->ckpt[sg + 1] : A->P[1];
    // Steps ckpt[sg] -> out through W[0] / W[1] (ckpt[sg] is only read).
    void *cur = A->W[0], *oth = A->W[1];
    if ((rc = advect_xy_moment(c, A->ckpt[sg], cur, 0.5 * dt, s))) return rc;
    for (int k = 0; k < len; ++k) {
      if ((rc = launch_field_poisson(c, s))) return rc;
      if ((rc = build_v_tables(c, dt, true, true, s))) return rc;
      if ((rc = advect_vxvy_any(c, cur, oth, &c->tab_vx, &c->tab_vy, s))) return rc;
      std::swap(cur, oth);
      if (k + 1 < len) {
        if ((rc = xy_xy_moment(c, cur, oth, out, s))) return rc;
        std::swap(cur, oth);
      }
    }
    StencilTable *tx = nullptr, *ty = nullptr;
    if ((rc = ensure_xy_table(c, 0, 0.5 * dt, &tx, s))) return rc;
    if ((rc = ensure_xy_table(c, 1, 0.5 * dt, &ty, s))) return rc;
    if ((rc = advect_xy_any(c, cur, out, tx, ty, s))) return rc;
  }
  if ((rc = energy_grad(A, A->P[1], A->L[0], s))) return rc;
  if (f_out) VLP4D_CUDA_TRY(cudaMemcpyAsync(f_out, A->P[1], A->fbytes, cudaMemcpyDeviceToDevice, s));
  return VLP4D_OK;
}

// Reverse sweep: per segment (last first) recompute the stage inputs a and
// fields E of its steps from the checkpoint, then run its reverse steps.
int backward_body(vlp4d_adjoint *A, void *grad, cudaStream_t s) {
  vlp4d_ctx *c = A->ctx;
  const double dt = c->dom.dt;
  const long long n2 = c->g.nxy();
  int rc;
  int cur = 0;
  const int nseg = A->store_all ? 1 : (int)A->ckpt.size();
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int len = A->nsteps - sg * A->every < A->every ? A->nsteps - sg * A->every : A->every;
    // The forward sweep stored everything when store_all.
    if (!A->store_all && (rc = store_segment(A, A->ckpt[sg], len, s))) return rc;
    // The reverse steps of the segment, last first.  Between two of them
    // the closing XY^T of one and the opening XY^T of the next are one pass
    // of the transposed 11-tap lines (as the forward sweep joins its x/y
    // half steps), so the adjoint state is materialised only at the
    // segment's start.  W[1] holds lb of the step, W[0] its la.
    if ((rc = advect_xy_any(c, A->L[cur], A->W[1], &A->tab_x_adj, &A->tab_y_adj, s))) return rc;
    for (int j = len - 1; j >= 0; --j) {
      if ((rc = reverse_core(A, A->seg[j], A->seg_e + 2 * (long long)c->fstride * j, A->W[1], A->W[0], s)))
        return rc;
      if (j > 0) {
        rc = A->tab_x11_adj.valid
                 ? launch_advect_xyxy_tables(c, A->W[0], A->W[1], &A->tab_x11_adj, &A->tab_y11_adj, false, s)
                 : VLP4D_ERR_UNSUPPORTED;
        if (rc == VLP4D_ERR_UNSUPPORTED) {
          if ((rc = advect_xy_any(c, A->W[0], A->L[cur ^ 1], &A->tab_x_adj, &A->tab_y_adj, s))) return rc;
          rc = advect_xy_any(c, A->L[cur ^ 1], A->W[1], &A->tab_x_adj, &A->tab_y_adj, s);
        }
        if (rc) return rc;
      } else {
        void *dst = sg == 0 ? grad : A->L[cur ^ 1];
        if ((rc = advect_xy_any(c, A->W[0], dst, &A->tab_x_adj, &A->tab_y_adj, s))) return rc;
        cur ^= 1;
      }
    }
  }
  return VLP4D_OK;
}

// Runs body(s) through a cached CUDA graph keyed by `key` (captured on the
// first call with that key); eager when graphs are off or a capture fails.
template <typename Body>
int run_graph(vlp4d_adjoint *A, cudaGraphExec_t &exec, const void **cached, const void *const *key, int nkey,
              cudaStream_t s, Body body) {
  if (!A->use_graphs) return body(s);
  bool hit = exec != nullptr;
  for (int i = 0; i < nkey && hit; ++i) hit = cached[i] == key[i];
  if (!hit) {
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    VLP4D_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    const int rc = body(s);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &g);
    cudaError_t ie = cudaErrorUnknown;
    if (rc == VLP4D_OK && e == cudaSuccess && g) ie = cudaGraphInstantiate(&exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (rc != VLP4D_OK || e != cudaSuccess || ie != cudaSuccess) {
      cudaGetLastError();
      exec = nullptr;
      A->use_graphs = false;
      return body(s);
    }
    for (int i = 0; i < nkey; ++i) cached[i] = key[i];
  }
  VLP4D_CUDA_TRY(cudaGraphLaunch(exec, s));
  return VLP4D_OK;
}

void destroy(vlp4d_adjoint *A) {
  if (!A) return;
  if (A->have_plan_g2) cufftDestroy(A->plan_g2);
  if (A->g_fwd) cudaGraphExecDestroy(A->g_fwd);
  if (A->g_bwd) cudaGraphExecDestroy(A->g_bwd);
  for (void *p : A->ckpt) cudaFree(p);
  for (void *p : A->seg) cudaFree(p);
  for (int i = 0; i < 2; ++i) {
    cudaFree(A->P[i]);
    cudaFree(A->W[i]);
    cudaFree(A->L[i]);
  }
  cudaFree(A->seg_e);
  cudaFree(A->gex);
  cudaFree(A->gpart);
  cudaFree(A->hx_hat);
  cudaFree(A->hy_hat);
  cudaFree(A->dw_vx);
  free_table(A->tab_x_adj);
  free_table(A->tab_y_adj);
  free_table(A->tab_vx_adj);
  free_table(A->tab_vy_adj);
  free_table(A->tab_x11_adj);
  free_table(A->tab_y11_adj);
  if (A->own) cudaStreamDestroy(A->own);
  delete A;
}

cudaStream_t pick_stream(vlp4d_adjoint *A, void *stream) {
  return stream ? (cudaStream_t)stream : A->own;
}

}  // namespace
}  // namespace vlp4d

using namespace vlp4d;

extern "C" {

int vlp4d_adjoint_create(vlp4d_ctx *ctx, int nsteps, int every, vlp4d_adjoint **out) {
  if (!out) return fail_msg(VLP4D_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (!ctx) return fail_msg(VLP4D_ERR_INVALID_ARG, "ctx is NULL");
  if (ctx->slab) return fail_msg(VLP4D_ERR_UNSUPPORTED, "adjoint_create: not available on a vy-slab context");
  if (nsteps < 1) return fail_msg(VLP4D_ERR_INVALID_ARG, "nsteps must be at least 1");
  if (every < 0) return fail_msg(VLP4D_ERR_INVALID_ARG, "the checkpoint interval must be at least 0");
  const bool store_all = every == 0;
  if (store_all || every > nsteps) every = nsteps;
  VLP4D_CUDA_TRY(cudaSetDevice(ctx->device));
  vlp4d_adjoint *A = new vlp4d_adjoint();
  A->ctx = ctx;
  A->nsteps = nsteps;
  A->every = every;
  A->store_all = store_all;
  A->fbytes = (size_t)ctx->g.cells() * ctx->elem;
  const char *g = getenv("VLP4D_ADJOINT_GRAPHS");
  if (g && *g == '0') A->use_graphs = false;
  const long long n2 = ctx->g.nxy();
  const int nh = (ctx->g.n[0] / 2 + 1) * ctx->g.n[1];
  auto bail = [&](int rc) {
    destroy(A);
    return rc;
  };
#define ADJ_ALLOC(ptr, bytes)                                                                      \
  do {                                                                                             \
    if (cudaMalloc((void **)&(ptr), (bytes)) != cudaSuccess) {                                     \
      cudaGetLastError();                                                                          \
      return bail(fail_msg(VLP4D_ERR_CUDA, "cudaMalloc failed in vlp4d_adjoint_create (" #ptr ")")); \
    }                                                                                              \
  } while (0)
  const int nck = store_all ? 0 : (nsteps + every - 1) / every;
  A->ckpt.assign(nck, nullptr);
  for (auto &p : A->ckpt) ADJ_ALLOC(p, A->fbytes);
  A->seg.assign(every, nullptr);
  for (auto &p : A->seg) ADJ_ALLOC(p, A->fbytes);
  for (int i = 0; i < 2; ++i) {
    ADJ_ALLOC(A->P[i], A->fbytes);
    ADJ_ALLOC(A->W[i], A->fbytes);
    ADJ_ALLOC(A->L[i], A->fbytes);
  }
  ADJ_ALLOC(A->seg_e, sizeof(double) * 2 * ctx->fstride * (size_t)every);
  ADJ_ALLOC(A->gex, sizeof(double) * (6 * n2 + 1));
  A->gey = A->gex + n2;
  A->lam_rho = A->gey + n2;
  A->save = A->lam_rho + n2;  // 3 * n2
  A->d_J = A->save + 3 * n2;
  A->gsegs = ctx->g.n[3] < 64 ? ctx->g.n[3] : 64;
  ADJ_ALLOC(A->gpart, sizeof(double) * 2 * n2 * (size_t)A->gsegs);
  ADJ_ALLOC(A->hx_hat, sizeof(cufftDoubleComplex) * nh);
  ADJ_ALLOC(A->hy_hat, sizeof(cufftDoubleComplex) * nh);
  ADJ_ALLOC(A->dw_vx, sizeof(double) * 12 * n2);
  A->dw_vy = A->dw_vx + 6 * n2;
#undef ADJ_ALLOC
  if (cudaStreamCreate(&A->own) != cudaSuccess) {
    cudaGetLastError();
    return bail(fail_msg(VLP4D_ERR_CUDA, "cudaStreamCreate failed"));
  }
  int rc;
  cudaStream_t s = A->own;
  if ((rc = build_xy_adj(ctx, 0, 0.5 * ctx->dom.dt, A->tab_x_adj, s))) return bail(rc);
  if ((rc = build_xy_adj(ctx, 1, 0.5 * ctx->dom.dt, A->tab_y_adj, s))) return bail(rc);
  if (xyxy_join(ctx)) {  // the joined reverse pass where the forward sweep joins too
    if ((rc = build_xy11_table(ctx, 0, 0.5 * ctx->dom.dt, true, A->tab_x11_adj, s))) return bail(rc);
    if ((rc = build_xy11_table(ctx, 1, 0.5 * ctx->dom.dt, true, A->tab_y11_adj, s))) return bail(rc);
  }
  if ((rc = alloc_table(A->tab_vx_adj, (int)n2))) return bail(rc);
  if ((rc = alloc_table(A->tab_vy_adj, (int)n2))) return bail(rc);
  A->tab_vx_adj.valid = A->tab_vy_adj.valid = true;
  if ((rc = alloc_table(ctx->tab_vx, (int)n2))) return bail(rc);
  if ((rc = alloc_table(ctx->tab_vy, (int)n2))) return bail(rc);
  // The forward x/y tables (host-built; their upload synchronises, which a
  // graph capture must not meet).
  StencilTable *t = nullptr;
  if ((rc = ensure_xy_table(ctx, 0, 0.5 * ctx->dom.dt, &t, s))) return bail(rc);
  if ((rc = ensure_xy_table(ctx, 1, 0.5 * ctx->dom.dt, &t, s))) return bail(rc);
  if (xyxy_join(ctx)) {
    if ((rc = ensure_xy11_table(ctx, 0, 0.5 * ctx->dom.dt, &t, s))) return bail(rc);
    if ((rc = ensure_xy11_table(ctx, 1, 0.5 * ctx->dom.dt, &t, s))) return bail(rc);
  }
  if ((rc = field_transpose_setup(A, s))) return bail(rc);
  *out = A;
  return VLP4D_OK;
}

int vlp4d_adjoint_destroy(vlp4d_adjoint *adj) {
  if (!adj) return VLP4D_OK;
  cudaSetDevice(adj->ctx->device);
  cudaDeviceSynchronize();
  destroy(adj);
  return VLP4D_OK;
}

int vlp4d_step_adjoint(vlp4d_adjoint *adj, const void *f_state, const void *lam_next, void *lam_out, void *stream) {
  if (!adj) return fail_msg(VLP4D_ERR_INVALID_ARG, "adj is NULL");
  if (!f_state || !lam_next || !lam_out) return fail_msg(VLP4D_ERR_INVALID_ARG, "NULL buffer");
  if (lam_out == lam_next || lam_out == f_state) return fail_msg(VLP4D_ERR_INVALID_ARG, "lam_out must be a separate buffer");
  return step_adjoint(adj, f_state, lam_next, lam_out, (cudaStream_t)stream);
}

int vlp4d_energy_grad(vlp4d_adjoint *adj, const void *f, double *J, void *lam, void *stream) {
  if (!adj) return fail_msg(VLP4D_ERR_INVALID_ARG, "adj is NULL");
  if (!f || !lam) return fail_msg(VLP4D_ERR_INVALID_ARG, "NULL buffer");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = energy_grad(adj, f, lam, s);
  if (rc) return rc;
  if (J) {
    VLP4D_CUDA_TRY(cudaMemcpyAsync(J, adj->d_J, sizeof(double), cudaMemcpyDeviceToHost, s));
    VLP4D_CUDA_TRY(cudaStreamSynchronize(s));
  }
  return VLP4D_OK;
}

int vlp4d_adjoint_forward(vlp4d_adjoint *adj, const void *f0, void *f_out, double *J, void *stream) {
  if (!adj) return fail_msg(VLP4D_ERR_INVALID_ARG, "adj is NULL");
  if (!f0) return fail_msg(VLP4D_ERR_INVALID_ARG, "f0 is NULL");
  vlp4d_adjoint *A = adj;
  cudaStream_t s = pick_stream(A, stream);
  A->have_forward = false;
  const void *key[2] = {f0, f_out};
  int rc = run_graph(A, A->g_fwd, A->k_fwd, key, 2, s,
                     [&](cudaStream_t st) { return forward_body(A, f0, f_out, st); });
  if (rc) return rc;
  VLP4D_CUDA_TRY(cudaMemcpyAsync(&A->J, A->d_J, sizeof(double), cudaMemcpyDeviceToHost, s));
  VLP4D_CUDA_TRY(cudaStreamSynchronize(s));
  if ((rc = vlp4d_check(A->ctx))) return rc;
  if (J) *J = A->J;
  A->have_forward = true;
  return VLP4D_OK;
}

int vlp4d_adjoint_backward(vlp4d_adjoint *adj, void *grad, void *stream) {
  if (!adj) return fail_msg(VLP4D_ERR_INVALID_ARG, "adj is NULL");
  if (!grad) return fail_msg(VLP4D_ERR_INVALID_ARG, "grad is NULL");
  vlp4d_adjoint *A = adj;
  if (!A->have_forward) return fail_msg(VLP4D_ERR_INVALID_ARG, "vlp4d_adjoint_backward needs a vlp4d_adjoint_forward first");
  cudaStream_t s = pick_stream(A, stream);
  const void *key[1] = {grad};
  int rc = run_graph(A, A->g_bwd, &A->k_bwd, key, 1, s, [&](cudaStream_t st) { return backward_body(A, grad, st); });
  if (rc) return rc;
  VLP4D_CUDA_TRY(cudaStreamSynchronize(s));
  return vlp4d_check(A->ctx);
}

}  // extern "C"
