// Fused x/y advection pass over (vx, vy) planes, with the velocity moment
// in its epilogue.
//
// Replaces advect_1D_x followed by advect_1D_y (miniapps/vlp4d/thrust/
// advection.hpp:77-201, run back to back in timestep.hpp:17-28) and, when
// requested, field_rho (field.cpp:6-32) of the result.
//
// Layout facts the kernel uses:
// * an (x, y) plane of f at fixed (ivx, ivy) is contiguous (nx*ny elements);
// * its x shift depends only on ivx and its y shift only on ivy, so one
//   x stencil and one y stencil (from the host-built line tables) serve
//   the whole plane.
// A CTA owns one chunk index c (output rows [c*R, (c+1)*R)) and walks planes
// g, g+G, g+2G, ...  For each plane it stages the R+5 input rows the chunk
// needs (rows c*R+my ... c*R+my+R+4 mod ny) into shared memory with 1D bulk
// copies (one per contiguous run; the periodic wrap splits a run in two), in
// a `stages`-deep mbarrier pipeline.  Phase X sweeps the R+5 rows along x
// into a shared buffer, phase Y sweeps that buffer along y and writes the R
// output rows with 16/32-byte vector stores.  Each input element is read from
// HBM once (halo rows of neighbouring chunks are reused through L2) and each
// output written once.  With the moment enabled, every CTA accumulates its
// chunk's outputs over its planes in FP64 shared memory and writes one
// partial per (plane group, cell); a second tiny kernel sums the groups.
#include "internal.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace vlp4d {

namespace {

constexpr int kBarBytes = 128;  // room for 16 mbarriers ahead of the buffers
constexpr int kMaxStages = 8;

struct PlaneArgs {
  const void *fin;
  void *fout;
  int nx, ny, nvx, nvy;
  int R;       // output rows per chunk (divides ny)
  int cpp;     // chunks per plane = ny / R
  int halo;    // 5 when the y sweep runs, else 0
  int stages;  // pipeline depth
  StencilTable tx, ty;
  double *rho_part;  // [G][nx*ny] partial moments, when the moment is fused
  int *err;
};

// Wraps a column index below 3*nx back into [0, nx) (two wraps happen only
// for nx = 4, where o0 + 8 = 8).
template <int NX>
__device__ __forceinline__ int wrap_col(int c, int nx) {
  if (NX && (NX & (NX - 1)) == 0) return c & (NX - 1);
  c = c >= nx ? c - nx : c;
  return c >= nx ? c - nx : c;
}

// Phase Y of one thread: RT outputs of its column quad from the RT+5 rows
// starting at src (stride nx), written in streaming order so that only a
// window of rows and differences is live; `emit(i, o)` receives row i.
template <int RT, typename Emit>
__device__ __forceinline__ void sweep_y(const double *src, int nx, const SweepW<double> &w, Emit emit) {
  double y[RT + 5][4];
#pragma unroll
  for (int j = 0; j < RT + 5; ++j) {
    load4(src + (size_t)j * nx, y[j]);
    if (j >= 5) {
      const int i = j - 5;
      double o[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        o[q] = interp6(w.w, y[i][q], y[i + 1][q], y[i + 2][q], y[i + 3][q], y[i + 4][q], y[j][q]);
      emit(i, o);
    }
  }
}
// FP32: columns (0,1) and (2,3) of the quad as packed pairs.
template <int RT, typename Emit>
__device__ __forceinline__ void sweep_y(const float *src, int nx, const SweepW<float> &w, Emit emit) {
  float2 y[RT + 5][2], d[RT + 4][2];
#pragma unroll
  for (int j = 0; j < RT + 5; ++j) {
    const float4 q4 = *reinterpret_cast<const float4 *>(src + (size_t)j * nx);
    y[j][0] = make_float2(q4.x, q4.y);
    y[j][1] = make_float2(q4.z, q4.w);
    if (j >= 1) {
#pragma unroll
      for (int h = 0; h < 2; ++h) d[j - 1][h] = sub2(y[j][h], y[j - 1][h]);
    }
    if (j >= 5) {
      const int i = j - 5;
      float2 o2[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) o2[h] = interp_diff2(w.v, y[i + 2][h], d[i][h], d[i + 1][h], d[i + 2][h], d[i + 3][h], d[i + 4][h]);
      const float o[4] = {o2[0].x, o2[0].y, o2[1].x, o2[1].y};
      emit(i, o);
    }
  }
}

// Stencil record of one line in shared memory: six weights (FP64, or the
// FP32 difference weights) and the tap offset, padded to 16-byte vectors.
template <typename T>
struct LineRec {
  T w[6];
  int m;
  int pad[sizeof(T) == 8 ? 3 : 1];
};
static_assert(sizeof(LineRec<float>) == 32 && sizeof(LineRec<double>) == 64, "line record layout");

template <typename T>
__device__ __forceinline__ void stage_lines(const StencilTable &t, int lines, LineRec<T> *dst) {
  const T *w = WeightsOf<T>::get(t);
  for (int l = threadIdx.x; l < lines; l += blockDim.x) {
#pragma unroll
    for (int k = 0; k < 6; ++k) dst[l].w[k] = w[6 * l + k];
    dst[l].m = t.m[l];
  }
}

template <typename T>
__device__ __forceinline__ int read_line(const LineRec<T> &r, T (&w)[6]) {
  LineRec<T> c = r;  // vector loads of the whole record
#pragma unroll
  for (int k = 0; k < 6; ++k) w[k] = c.w[k];
  return c.m;
}

// Error exit after a copy timed out: flag it, let the copies already issued
// for items it .. it+S-1 land (bounded waits), then leave.
__device__ __noinline__ void plane_abort(const PlaneArgs &a, uint64_t *bars, long long it, long long n_items, int S,
                                         long long issued_end = -1) {
  if (threadIdx.x == 0) {
    atomicExch(a.err, 1);
    const long long end = issued_end >= 0 ? issued_end : it + S;
    const long long last = n_items < end ? n_items : end;
    for (long long k = it; k < last; ++k) mbar_wait_bounded(&bars[k % S], (uint32_t)((k / S) & 1));
  }
  __syncthreads();
}

// Template parameters: element type, row width (0 = runtime a.nx), output
// rows per thread in the y phase, which sweeps run, moment epilogue, and
// INPLACE (x and y both on, nx/4 dividing 32): phase X writes the x-swept
// rows back into the staged slot instead of a separate tile.  A row's
// column quads then all belong to one warp, which reads the whole row
// before any lane writes it (__syncwarp); phase Y reads the slot; the slot
// of item it - 1 is refilled at the barrier of item it (one item later than
// with the separate tile).  Without the two x-swept tiles an FP64 pass at
// 128^4 fits two CTAs per SM.
// FP64 pair mapping of k_plane.  x6_pair_row: the x-swept outputs (c, c + 1)
// of a row from the eight values at the even column a0 = (c + mx) - r, a0
// + 1, ... (periodic; the row width is even); output q uses t[r+q ..
// r+q+5], computed as x4_from<double> computes it.  sweep_y_pairs: phase Y
// of the columns (c, c + 1, c + h, c + h + 1) from RT + 5 rows, each output
// as sweep_y<double> computes it.
template <int R_>
__device__ __forceinline__ void x6_pair_from(const double (&t)[8], const SweepW<double> &w, double (&o)[2]) {
#pragma unroll
  for (int q = 0; q < 2; ++q)
    o[q] = interp6(w.w, t[R_ + q], t[R_ + q + 1], t[R_ + q + 2], t[R_ + q + 3], t[R_ + q + 4], t[R_ + q + 5]);
}
__device__ __forceinline__ void x6_pair_row(const double *row, int a0, int nx, int r, const SweepW<double> &w,
                                            double (&o)[2]) {
  double t[8];
  int c = a0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const double2 v = *reinterpret_cast<const double2 *>(row + c);
    t[2 * j] = v.x;
    t[2 * j + 1] = v.y;
    c += 2;
    if (c >= nx) c -= nx;
  }
  if (r) x6_pair_from<1>(t, w, o);
  else x6_pair_from<0>(t, w, o);
}
template <int RT, typename Emit>
__device__ __forceinline__ void sweep_y_pairs(const double *src, int nx, int h, const SweepW<double> &w, Emit emit) {
  double y[RT + 5][4];
#pragma unroll
  for (int j = 0; j < RT + 5; ++j) {
    const double2 lo = *reinterpret_cast<const double2 *>(src + (size_t)j * nx);
    const double2 hi = *reinterpret_cast<const double2 *>(src + (size_t)j * nx + h);
    y[j][0] = lo.x;
    y[j][1] = lo.y;
    y[j][2] = hi.x;
    y[j][3] = hi.y;
    if (j >= 5) {
      const int i = j - 5;
      double o[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        o[q] = interp6(w.w, y[i][q], y[i + 1][q], y[i + 2][q], y[i + 3][q], y[i + 4][q], y[j][q]);
      emit(i, o);
    }
  }
}

// Thread t owns column quad c0 = 4*(t % (nx/4)) and row group t / (nx/4)
// for the whole kernel; blockDim = (nx/4) * (R/RT).
template <typename T, int NX, int RT, bool DX, bool DY, bool RHO, bool INPLACE = false>
__global__ void __launch_bounds__(512) k_plane(PlaneArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int nx = NX ? NX : a.nx;
  const int ny = a.ny, R = a.R, S = a.stages;
  const int vrows = R + (DY ? 5 : 0);
  const int ncg = nx >> 2;
  const size_t slot_elems = (size_t)vrows * nx;
  const uint32_t slot_bytes = (uint32_t)(slot_elems * sizeof(T));
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  // Stencil records of every x line (by ivx) and y line (by ivy).
  LineRec<T> *xrec = reinterpret_cast<LineRec<T> *>(smem + kBarBytes);
  LineRec<T> *yrec = xrec + (DX ? a.nvx : 0);
  T *slots = reinterpret_cast<T *>(yrec + (DY ? a.nvy : 0));
  // Two x-swept buffers (x and y both on): item it writes xs[it & 1], so the
  // only barrier per item is the one between phase X and phase Y.
  T *xs_base = slots + (size_t)S * slot_elems;  // unused when INPLACE

  const int cg = threadIdx.x % ncg;
  const int rg = threadIdx.x / ncg;
  const int RG = blockDim.x / ncg;  // row groups; R == RG * RT
  const int c0 = cg * 4;
  // FP64: the thread's four columns are the pairs (yc, yc + 1) and
  // (yc + nx/2, yc + nx/2 + 1), so that a warp's 16-byte shared-memory
  // accesses are consecutive (a quad of doubles per lane would put two
  // lanes of each quarter-warp phase on the same banks).
  constexpr bool PAIRS = sizeof(T) == 8;
  const int yc = cg * 2;
  const int hx = nx >> 1;
  const int r0 = rg * RT;

  const int chunk = blockIdx.x % a.cpp;
  const int G = gridDim.x / a.cpp;
  const int g = blockIdx.x / a.cpp;
  const long long planes = (long long)a.nvx * a.nvy;
  const long long n_items = g < planes ? (planes - g + G - 1) / G : 0;
  const long long plane_elems = (long long)nx * ny;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  if (DX) stage_lines<T>(a.tx, a.nvx, xrec);
  if (DY) stage_lines<T>(a.ty, a.nvy, yrec);
  __syncthreads();

  // Thread 0: stage the input rows of item `it` into its slot.
  auto issue = [&](long long it) {
    const long long p = g + it * G;
    int phys = chunk * R;
    if (DY) {
      phys += yrec[(int)(p / a.nvx)].m;
      if (phys >= ny) phys -= ny;
    }
    uint64_t *bar = &bars[it % S];
    mbar_arrive_expect_tx(bar, slot_bytes);
    const T *src = static_cast<const T *>(a.fin) + p * plane_elems;
    T *dst = slots + (size_t)(it % S) * slot_elems;
    int remaining = vrows;
    while (remaining > 0) {
      const int len = remaining < ny - phys ? remaining : ny - phys;
      bulk_load(dst, src + (long long)phys * nx, (uint32_t)((size_t)len * nx * sizeof(T)), bar);
      dst += (size_t)len * nx;
      remaining -= len;
      phys = 0;
    }
  };
  if (threadIdx.x == 0) {
    const long long pre = n_items < S ? n_items : S;
    for (long long it = 0; it < pre; ++it) issue(it);
  }

  double racc[RHO ? RT : 1][4];
#pragma unroll
  for (int i = 0; i < (RHO ? RT : 1); ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) racc[i][q] = 0.0;

  // Plane index p = g + it*G, tracked as (ivx, ivy) without divisions.
  const int gdx = G % a.nvx, gdy = G / a.nvx;
  int ivx = g % a.nvx, ivy = g / a.nvx;
  int slot = 0;          // it % S
  uint32_t parity = 0;   // (it / S) & 1
  for (long long it = 0; it < n_items; ++it) {
    const bool ok = mbar_wait_bounded(&bars[slot], parity);
    const long long p = g + it * G;
    const T *in = slots + (size_t)slot * slot_elems;
    T *outp = static_cast<T *>(a.fout) + p * plane_elems + (long long)chunk * R * nx;
    T *xs = xs_base + (size_t)(it & 1) * slot_elems;

    if (DX) {  // Phase X: staged rows rg, rg+RG, ...; this thread's column quad.
      T wl[6];
      const int mx = read_line(xrec[ivx], wl);
      int base = c0 + mx;
      SweepW<T> wx;
      make_sweep_w(wl, wx);
      base = wrap_col<NX>(base, nx);
      const int rr = base & 3;
      const int o0 = base - rr, o1 = wrap_col<NX>(o0 + 4, nx), o2 = wrap_col<NX>(o0 + 8, nx);
      // Pair mapping: the tap windows of the pairs at yc and yc + nx/2
      // start at the even columns pa and pb, offset pr within them.
      int pa = wrap_col<NX>(yc + mx, nx);
      const int pr = pa & 1;
      pa -= pr;
      const int pb = pa + hx >= nx ? pa - hx : pa + hx;
      if constexpr (PAIRS) {
        const int rgw = (int)((threadIdx.x & ~31u) / (unsigned)ncg);
        const int trips = INPLACE ? (vrows - rgw + RG - 1) / RG : 0;
        const unsigned wlane = blockDim.x - (threadIdx.x & ~31u);
        const unsigned wmask = wlane >= 32 ? 0xffffffffu : (1u << wlane) - 1u;
        const int nv = INPLACE ? trips : (vrows - rg + RG - 1) / RG;
        for (int k = 0; k < nv; ++k) {
          const int v = rg + k * RG;
          T *row = const_cast<T *>(in) + (size_t)v * nx;
          double oa[2], ob[2];
          if (v < vrows) {
            x6_pair_row(row, pa, nx, pr, wx, oa);
            x6_pair_row(row, pb, nx, pr, wx, ob);
          }
          T *dst;
          if constexpr (INPLACE) {
            __syncwarp(wmask);  // the row is read by all its lanes
            dst = row;
          } else {
            dst = (DY ? xs : outp) + (size_t)v * nx;
          }
          if (v < vrows) {
            *reinterpret_cast<double2 *>(dst + yc) = make_double2(oa[0], oa[1]);
            *reinterpret_cast<double2 *>(dst + yc + hx) = make_double2(ob[0], ob[1]);
          }
        }
        if constexpr (INPLACE) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      } else if constexpr (INPLACE) {
        // Trip count of the warp's first row group, so that every lane
        // reaches each __syncwarp.
        const int rgw = (int)((threadIdx.x & ~31u) / (unsigned)ncg);
        const int trips = (vrows - rgw + RG - 1) / RG;
        // The lanes this warp has (small grids give blocks below 32 threads).
        const unsigned wl = blockDim.x - (threadIdx.x & ~31u);
        const unsigned wmask = wl >= 32 ? 0xffffffffu : (1u << wl) - 1u;
        for (int k = 0; k < trips; ++k) {
          const int v = rg + k * RG;
          T *row = const_cast<T *>(in) + (size_t)v * nx;
          T t[12], q4[4], o[4];
          if (v < vrows) {
            load4(row + o0, q4);
            t[0] = q4[0]; t[1] = q4[1]; t[2] = q4[2]; t[3] = q4[3];
            load4(row + o1, q4);
            t[4] = q4[0]; t[5] = q4[1]; t[6] = q4[2]; t[7] = q4[3];
            load4(row + o2, q4);
            t[8] = q4[0]; t[9] = q4[1]; t[10] = q4[2]; t[11] = q4[3];
            sweep_x4(t, rr, wx, o);
          }
          __syncwarp(wmask);  // the row is read by all its lanes
          if (v < vrows) store4(row + c0, o);
        }
        // These generic writes precede the slot's next bulk copy.
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      } else {
        for (int v = rg; v < vrows; v += RG) {
          const T *row = in + (size_t)v * nx;
          T t[12], q4[4];
          load4(row + o0, q4);
          t[0] = q4[0]; t[1] = q4[1]; t[2] = q4[2]; t[3] = q4[3];
          load4(row + o1, q4);
          t[4] = q4[0]; t[5] = q4[1]; t[6] = q4[2]; t[7] = q4[3];
          load4(row + o2, q4);
          t[8] = q4[0]; t[9] = q4[1]; t[10] = q4[2]; t[11] = q4[3];
          T o[4];
          sweep_x4(t, rr, wx, o);
          if (DY) {
            store4(xs + (size_t)v * nx + c0, o);
          } else {
            store4(outp + (size_t)v * nx + c0, o);
          }
        }
      }
    }
    if (DX && DY) {
      if constexpr (INPLACE) {
        // The x-swept rows are complete; every thread is done with item
        // it - 1, whose slot now takes item it - 1 + S.
        const long long issued_end = it == 0 ? (long long)S : it - 1 + S;
        if (__syncthreads_or(!ok)) {
          plane_abort(a, bars, it, n_items, S, issued_end);
          return;
        }
        if (threadIdx.x == 0 && it > 0 && it - 1 + S < n_items) issue(it - 1 + S);
      } else {
        // xs is complete and the staged slot is no longer read: refill it.
        if (__syncthreads_or(!ok)) {
          plane_abort(a, bars, it, n_items, S);
          return;
        }
        if (threadIdx.x == 0 && it + S < n_items) issue(it + S);
      }
    }
    if (DY) {  // Phase Y: rows r0 .. r0+RT-1 of this thread's column quad.
      T wl[6];
      read_line(yrec[ivy], wl);
      SweepW<T> wy;
      make_sweep_w(wl, wy);
      if constexpr (PAIRS) {
        const double *src = ((DX && !INPLACE) ? xs : in) + (size_t)r0 * nx + yc;
        T *dst = outp + (size_t)r0 * nx + yc;
        sweep_y_pairs<RT>(src, nx, hx, wy, [&](int i, const double (&o)[4]) {
          *reinterpret_cast<double2 *>(dst + (size_t)i * nx) = make_double2(o[0], o[1]);
          *reinterpret_cast<double2 *>(dst + (size_t)i * nx + hx) = make_double2(o[2], o[3]);
          if (RHO) {
#pragma unroll
            for (int q = 0; q < 4; ++q) racc[i][q] += o[q];
          }
        });
      } else {
        const T *src = ((DX && !INPLACE) ? xs : in) + (size_t)r0 * nx + c0;
        T *dst = outp + (size_t)r0 * nx + c0;
        sweep_y<RT>(src, nx, wy, [&](int i, const T (&o)[4]) {
          store4(dst + (size_t)i * nx, o);
          if (RHO) {
#pragma unroll
            for (int q = 0; q < 4; ++q) racc[i][q] += (double)o[q];
          }
        });
      }
    }
    ivx += gdx;
    ivy += gdy;
    if (ivx >= a.nvx) {
      ivx -= a.nvx;
      ++ivy;
    }
    if (++slot == S) {
      slot = 0;
      parity ^= 1u;
    }
    if (DX && DY) continue;
    // One sweep only: the slot is free once every thread is here.
    if (__syncthreads_or(!ok)) {
      plane_abort(a, bars, it, n_items, S);
      return;
    }
    if (threadIdx.x == 0 && it + S < n_items) issue(it + S);
  }
  if (RHO) {
    double *dst = a.rho_part + (long long)g * plane_elems + ((long long)chunk * R + r0) * nx + (PAIRS ? yc : c0);
    const int second = PAIRS ? hx : 2;  // element offset of the second double pair
#pragma unroll
    for (int i = 0; i < RT; ++i) {
      *reinterpret_cast<double2 *>(dst + (size_t)i * nx) = make_double2(racc[i][0], racc[i][1]);
      *reinterpret_cast<double2 *>(dst + (size_t)i * nx + second) = make_double2(racc[i][2], racc[i][3]);
    }
  }
}

// Two consecutive x/y half steps in one pass: the closing x, y half step of
// one Strang step and the opening one of the next, which no field solve
// separates.  Two x shifts by the same dt are one 11-tap x stencil (offset
// 2m mod nx, weights w * w), likewise in y, and the x and y shifts commute
// exactly (their weights depend on different indices), so
//   y x y x = (y y)(x x):   Y11 on the staged rows, then X11,
// which equals the four sweeps in exact arithmetic and in floating point up
// to rounding.  Per item: stage the R + 10 input rows the chunk needs,
// Y11 (thread: RT output rows of its column quad) into a double-buffered
// shared tile, one barrier, X11 of the thread's rows to the output, with the
// moment of the result in FP64 registers as in k_plane.
template <typename T>
struct LineRec11;
template <>
struct LineRec11<float> {
  float w[11];  // difference weights u[0..9] (u[10] unused)
  int m;
};
template <>
struct LineRec11<double> {
  double w[11];
  int m;
  int pad;
};
static_assert(sizeof(LineRec11<float>) == 48 && sizeof(LineRec11<double>) == 96, "11-tap record layout");

template <typename T>
__device__ __forceinline__ void stage_lines11(const StencilTable &t, int lines, LineRec11<T> *dst) {
  for (int l = threadIdx.x; l < lines; l += blockDim.x) {
#pragma unroll
    for (int k = 0; k < 11; ++k) dst[l].w[k] = sizeof(T) == 4 ? (T)t.wf[11 * l + k] : (T)t.w[11 * l + k];
    dst[l].m = t.m[l];
  }
}

// FP32: weights as packed pairs (u_j, u_j); FP64: the 11 weights.
template <typename T>
struct W11 {
  T w[11];
};
template <>
struct W11<float> {
  float2 u[10];
};
__device__ __forceinline__ int read_line11(const LineRec11<float> &r, W11<float> &w) {
  LineRec11<float> c = r;
#pragma unroll
  for (int k = 0; k < 10; ++k) w.u[k] = make_float2(c.w[k], c.w[k]);
  return c.m;
}
__device__ __forceinline__ int read_line11(const LineRec11<double> &r, W11<double> &w) {
  LineRec11<double> c = r;
#pragma unroll
  for (int k = 0; k < 11; ++k) w.w[k] = c.w[k];
  return c.m;
}

// out = f_5 + sum_j u_j d_j on packed pairs (d_j = f_{j+1} - f_j).
__device__ __forceinline__ float2 interp11_2(const float2 (&u)[10], float2 f5, const float2 *d) {
  float2 acc = __fmul2_rn(u[0], d[0]);
#pragma unroll
  for (int j = 1; j < 10; ++j) acc = __ffma2_rn(u[j], d[j], acc);
  return __fadd2_rn(f5, acc);
}

// Y11 of one thread: RT output rows of its column quad from the RT + 10
// rows starting at src (stride nx), streamed; emit(i, o) receives row i.
template <int RT, typename Emit>
__device__ __forceinline__ void sweep_y11(const float *src, int nx, const W11<float> &w, Emit emit) {
  float2 y[RT + 10][2], d[RT + 9][2];
#pragma unroll
  for (int j = 0; j < RT + 10; ++j) {
    const float4 q4 = *reinterpret_cast<const float4 *>(src + (size_t)j * nx);
    y[j][0] = make_float2(q4.x, q4.y);
    y[j][1] = make_float2(q4.z, q4.w);
    if (j >= 1) {
#pragma unroll
      for (int h = 0; h < 2; ++h) d[j - 1][h] = sub2(y[j][h], y[j - 1][h]);
    }
    if (j >= 10) {
      const int i = j - 10;
      float2 o2[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float2 dd[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) dd[k] = d[i + k][h];
        o2[h] = interp11_2(w.u, y[i + 5][h], dd);
      }
      const float o[4] = {o2[0].x, o2[0].y, o2[1].x, o2[1].y};
      emit(i, o);
    }
  }
}
template <int RT, typename Emit>
__device__ __forceinline__ void sweep_y11(const double *src, int nx, const W11<double> &w, Emit emit) {
  double y[RT + 10][4];
#pragma unroll
  for (int j = 0; j < RT + 10; ++j) {
    load4(src + (size_t)j * nx, y[j]);
    if (j >= 10) {
      const int i = j - 10;
      double o[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double acc = w.w[0] * y[i][q];
#pragma unroll
        for (int k = 1; k < 11; ++k) acc = fma(w.w[k], y[i + k][q], acc);
        o[q] = acc;
      }
      emit(i, o);
    }
  }
}

// X11 of four outputs from the twenty values t[0..19] starting at the
// aligned column a0 = c0 + mx - r (output q uses t[r+q .. r+q+10]).
template <int R_>
__device__ __forceinline__ void x11_from(const float (&t)[20], const W11<float> &w, float (&o)[4]) {
  float d[13];
#pragma unroll
  for (int j = 0; j < 13; ++j) d[j] = t[R_ + j + 1] - t[R_ + j];
  float2 dp[12];
#pragma unroll
  for (int j = 0; j < 12; ++j) dp[j] = make_float2(d[j], d[j + 1]);
  const float2 lo = interp11_2(w.u, make_float2(t[R_ + 5], t[R_ + 6]), dp);
  const float2 hi = interp11_2(w.u, make_float2(t[R_ + 7], t[R_ + 8]), dp + 2);
  o[0] = lo.x;
  o[1] = lo.y;
  o[2] = hi.x;
  o[3] = hi.y;
}
template <int R_>
__device__ __forceinline__ void x11_from(const double (&t)[20], const W11<double> &w, double (&o)[4]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double acc = w.w[0] * t[R_ + q];
#pragma unroll
    for (int k = 1; k < 11; ++k) acc = fma(w.w[k], t[R_ + q + k], acc);
    o[q] = acc;
  }
}
// X11 of eight outputs from t[0..23] (FP32): the two quads' loads, column
// differences and register pairs are shared; each output is computed
// exactly as x11_from computes it.
template <int R_>
__device__ __forceinline__ void x11_from8(const float (&t)[24], const W11<float> &w, float (&o)[8]) {
  float d[17];
#pragma unroll
  for (int j = 0; j < 17; ++j) d[j] = t[R_ + j + 1] - t[R_ + j];
  float2 dp[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) dp[j] = make_float2(d[j], d[j + 1]);
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const float2 r = interp11_2(w.u, make_float2(t[R_ + 5 + 2 * p], t[R_ + 6 + 2 * p]), dp + 2 * p);
    o[2 * p] = r.x;
    o[2 * p + 1] = r.y;
  }
}
__device__ __forceinline__ void sweep_x11_8(const float (&t)[24], int r, const W11<float> &w, float (&o)[8]) {
  switch (r) {
    case 0: x11_from8<0>(t, w, o); break;
    case 1: x11_from8<1>(t, w, o); break;
    case 2: x11_from8<2>(t, w, o); break;
    default: x11_from8<3>(t, w, o); break;
  }
}

template <typename T>
__device__ __forceinline__ void sweep_x11(const T (&t)[20], int r, const W11<T> &w, T (&o)[4]) {
  switch (r) {
    case 0: x11_from<0>(t, w, o); break;
    case 1: x11_from<1>(t, w, o); break;
    case 2: x11_from<2>(t, w, o); break;
    default: x11_from<3>(t, w, o); break;
  }
}

// X8 (FP32, RT = 4, nx a multiple of 8): the X11 phase maps thread t to
// the column octet 8*(t mod nx/8) and the two rows 2*(t / (nx/8)) + {0, 1}
// of the chunk (as many threads as the Y11 mapping), so that neighbouring
// outputs share their loads, differences and register pairs.  Its 16-byte
// loads of neighbouring lanes lie 32 bytes apart, which would put two lanes
// of each quarter-warp phase on the same banks; the intermediate tile
// therefore stores 16-byte chunk c of a row at chunk c ^ ((c >> 3) & 1),
// which maps the eight chunks one phase reads (2t + s for t = 0..7, any s)
// to eight different bank groups, and keeps the Y11 stores (eight
// consecutive chunks per phase) conflict-free.
__device__ __forceinline__ int xyxy_swz(int chunk) { return chunk ^ ((chunk >> 3) & 1); }
// RHO = false: no moment (the reverse mode's joined pass of transposed
// stencils has no use for one).
template <typename T, int NX, int RT, bool X8 = false, bool RHO = true>
__global__ void __launch_bounds__(512) k_plane_xyxy(PlaneArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int nx = NX ? NX : a.nx;
  const int ny = a.ny, R = a.R, S = a.stages;
  const int ncg = nx >> 2;
  const size_t slot_elems = (size_t)(R + 10) * nx;
  const uint32_t slot_bytes = (uint32_t)(slot_elems * sizeof(T));
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  LineRec11<T> *xrec = reinterpret_cast<LineRec11<T> *>(smem + kBarBytes);
  LineRec11<T> *yrec = xrec + a.nvx;
  T *slots = reinterpret_cast<T *>(yrec + a.nvy);
  T *ys_base = slots + (size_t)S * slot_elems;  // two R-row tiles

  const int cg = threadIdx.x % ncg;
  const int rg = threadIdx.x / ncg;
  const int c0 = cg * 4;
  const int r0 = rg * RT;
  const int chunk = blockIdx.x % a.cpp;
  const int G = gridDim.x / a.cpp;
  const int g = blockIdx.x / a.cpp;
  const long long planes = (long long)a.nvx * a.nvy;
  const long long n_items = g < planes ? (planes - g + G - 1) / G : 0;
  const long long plane_elems = (long long)nx * ny;

  if (threadIdx.x == 0) {
    for (int st = 0; st < S; ++st) mbar_init(&bars[st], 1);
    mbar_fence_init();
  }
  stage_lines11<T>(a.tx, a.nvx, xrec);
  stage_lines11<T>(a.ty, a.nvy, yrec);
  __syncthreads();

  auto issue = [&](long long it) {
    const long long p = g + it * G;
    int phys = (chunk * R + yrec[(int)(p / a.nvx)].m) % ny;
    uint64_t *bar = &bars[it % S];
    mbar_arrive_expect_tx(bar, slot_bytes);
    const T *src = static_cast<const T *>(a.fin) + p * plane_elems;
    T *dst = slots + (size_t)(it % S) * slot_elems;
    int remaining = R + 10;
    while (remaining > 0) {
      const int len = remaining < ny - phys ? remaining : ny - phys;
      bulk_load(dst, src + (long long)phys * nx, (uint32_t)((size_t)len * nx * sizeof(T)), bar);
      dst += (size_t)len * nx;
      remaining -= len;
      phys = 0;
    }
  };
  if (threadIdx.x == 0) {
    const long long pre = n_items < S ? n_items : S;
    for (long long it = 0; it < pre; ++it) issue(it);
  }

  double racc[RT][4];
#pragma unroll
  for (int i = 0; i < RT; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) racc[i][q] = 0.0;
  // X8 mapping (racc[2 * i + h][q] holds row i, column c8 + 4h + q).
  const int c8 = X8 ? 8 * (threadIdx.x % (nx >> 3)) : 0;
  const int r8 = X8 ? 2 * (threadIdx.x / (nx >> 3)) : 0;

  const int gdx = G % a.nvx, gdy = G / a.nvx;
  int ivx = g % a.nvx, ivy = g / a.nvx;
  int slot = 0;
  uint32_t parity = 0;
  for (long long it = 0; it < n_items; ++it) {
    const bool ok = mbar_wait_bounded(&bars[slot], parity);
    const long long p = g + it * G;
    const T *in = slots + (size_t)slot * slot_elems;
    T *ys = ys_base + (size_t)(it & 1) * R * nx;
    T *outp = static_cast<T *>(a.fout) + p * plane_elems + (long long)chunk * R * nx;
    {  // Y11: rows r0 .. r0+RT-1 of this thread's column quad.
      W11<T> wy;
      read_line11(yrec[ivy], wy);
      sweep_y11<RT>(in + (size_t)r0 * nx + c0, nx, wy,
                    [&](int i, const T (&o)[4]) {
                      const int cs = X8 ? 4 * xyxy_swz(c0 >> 2) : c0;
                      store4(ys + (size_t)(r0 + i) * nx + cs, o);
                    });
    }
    // ys is complete and the staged slot is no longer read: refill it.
    if (__syncthreads_or(!ok)) {
      plane_abort(a, bars, it, n_items, S);
      return;
    }
    if (threadIdx.x == 0 && it + S < n_items) issue(it + S);
    if constexpr (X8) {  // X11 of the thread's column octet and two rows, the moment.
      W11<T> wx;
      int base = c8 + read_line11(xrec[ivx], wx);
      base = base % nx;
      const int rr = base & 3;
      int o[6];
      o[0] = base - rr;
#pragma unroll
      for (int k = 1; k < 6; ++k) {
        o[k] = o[k - 1] + 4;
        if (o[k] >= nx) o[k] -= nx;
      }
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const T *row = ys + (size_t)(r8 + i) * nx;
        float t[24], q4[4];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          load4(row + 4 * xyxy_swz(o[k] >> 2), q4);
          t[4 * k] = q4[0];
          t[4 * k + 1] = q4[1];
          t[4 * k + 2] = q4[2];
          t[4 * k + 3] = q4[3];
        }
        float out[8];
        sweep_x11_8(t, rr, wx, out);
        const float lo[4] = {out[0], out[1], out[2], out[3]}, hi[4] = {out[4], out[5], out[6], out[7]};
        store4(outp + (size_t)(r8 + i) * nx + c8, lo);
        store4(outp + (size_t)(r8 + i) * nx + c8 + 4, hi);
        if constexpr (RHO) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            racc[2 * i][q] += (double)lo[q];
            racc[2 * i + 1][q] += (double)hi[q];
          }
        }
      }
    } else {  // X11 of the thread's rows, the moment.
      W11<T> wx;
      int base = c0 + read_line11(xrec[ivx], wx);
      base = base % nx;
      const int rr = base & 3;
      int o[5];
      o[0] = base - rr;
#pragma unroll
      for (int k = 1; k < 5; ++k) {
        o[k] = o[k - 1] + 4;
        if (o[k] >= nx) o[k] -= nx;
      }
#pragma unroll
      for (int i = 0; i < RT; ++i) {
        const T *row = ys + (size_t)(r0 + i) * nx;
        T t[20], q4[4];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
          load4(row + o[k], q4);
          t[4 * k] = q4[0];
          t[4 * k + 1] = q4[1];
          t[4 * k + 2] = q4[2];
          t[4 * k + 3] = q4[3];
        }
        T out[4];
        sweep_x11(t, rr, wx, out);
        store4(outp + (size_t)(r0 + i) * nx + c0, out);
        if constexpr (RHO) {
#pragma unroll
          for (int q = 0; q < 4; ++q) racc[i][q] += (double)out[q];
        }
      }
    }
    ivx += gdx;
    ivy += gdy;
    if (ivx >= a.nvx) {
      ivx -= a.nvx;
      ++ivy;
    }
    if (++slot == S) {
      slot = 0;
      parity ^= 1u;
    }
  }
  if constexpr (!RHO) {
    return;
  } else if constexpr (X8) {
    double *rdst = a.rho_part + (long long)g * plane_elems + ((long long)chunk * R + r8) * nx + c8;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        double2 *p2 = reinterpret_cast<double2 *>(rdst + (size_t)i * nx + 4 * h);
        p2[0] = make_double2(racc[2 * i + h][0], racc[2 * i + h][1]);
        p2[1] = make_double2(racc[2 * i + h][2], racc[2 * i + h][3]);
      }
  } else {
    double *rdst = a.rho_part + (long long)g * plane_elems + ((long long)chunk * R + r0) * nx + c0;
#pragma unroll
    for (int i = 0; i < RT; ++i) {
      reinterpret_cast<double2 *>(rdst + (size_t)i * nx)[0] = make_double2(racc[i][0], racc[i][1]);
      reinterpret_cast<double2 *>(rdst + (size_t)i * nx)[1] = make_double2(racc[i][2], racc[i][3]);
    }
  }
}

// FP64 form of the two-half-step pass for row widths a warp holds whole
// (nx/4 divides 32).  With 1 KB rows the FP32 structure (staged rows, a Y11
// tile, X11) leaves one CTA per SM; here, as in k_plane's in-place FP64
// pass, the staged slot is swept in place:
//   X11: each warp sweeps whole staged rows (all R + 10 of them) and writes
//        the x-swept row back over itself after every lane has read it;
//   one CTA barrier;
//   Y11: thread (quad cg, row group rg) streams its RT + 10 x-swept rows
//        down the slot and accumulates each row into the RT outputs it
//        belongs to (out_i = sum_k W_k row_{i+k}), so only RT accumulators
//        and one row are live; each finished output goes to global memory
//        and into the FP64 moment.
// X11 then Y11 applies the same two composed stencils as Y11 then X11 (they
// commute), at the cost of X11 on the 10 halo rows.  The slot of item it is
// read until Y11(it) ends, so it is refilled at the barrier of item it + 1
// (two stages keep two CTAs per SM at 128^4).  Weights plain (FP64 sums
// w * w of the per-line Lagrange weights, as k_plane_xyxy<double>).
// X11 of the output pair (c, c + 1) of an FP64 row, from the fourteen
// values at the even column a0 = (c + mx) - r, a0 + 1, ... (periodic; the
// row width is even): output q uses t[r+q .. r+q+10], each computed as
// x11_from<double> computes it.
template <int R_>
__device__ __forceinline__ void x11_pair_from(const double (&t)[14], const W11<double> &w, double (&o)[2]) {
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    double acc = w.w[0] * t[R_ + q];
#pragma unroll
    for (int k = 1; k < 11; ++k) acc = fma(w.w[k], t[R_ + q + k], acc);
    o[q] = acc;
  }
}
__device__ __forceinline__ void x11_pair_row(const double *row, int a0, int nx, int r, const W11<double> &w,
                                             double (&o)[2]) {
  double t[14];
  int c = a0;
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    const double2 v = *reinterpret_cast<const double2 *>(row + c);
    t[2 * j] = v.x;
    t[2 * j + 1] = v.y;
    c += 2;
    if (c >= nx) c -= nx;
  }
  if (r) x11_pair_from<1>(t, w, o);
  else x11_pair_from<0>(t, w, o);
}

template <int NX, int RT, bool RHO = true>
__global__ void __launch_bounds__(512) k_plane_xyxy64(PlaneArgs a) {
  using T = double;
  extern __shared__ __align__(128) unsigned char smem[];
  const int nx = NX ? NX : a.nx;
  const int ny = a.ny, R = a.R, S = a.stages;
  const int vrows = R + 10;
  const int ncg = nx >> 2;
  const size_t slot_elems = (size_t)vrows * nx;
  const uint32_t slot_bytes = (uint32_t)(slot_elems * sizeof(T));
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  LineRec11<T> *xrec = reinterpret_cast<LineRec11<T> *>(smem + kBarBytes);
  LineRec11<T> *yrec = xrec + a.nvx;
  T *slots = reinterpret_cast<T *>(yrec + a.nvy);

  const int cg = threadIdx.x % ncg;
  const int rg = threadIdx.x / ncg;
  const int RG = blockDim.x / ncg;  // row groups; R == RG * RT
  const int c0 = cg * 4;  // X11: the column quad c0 .. c0+3
  const int yc = cg * 2;  // Y11 and the moment: columns yc, yc+1 and yc+nx/2, yc+nx/2+1
  const int r0 = rg * RT;
  const int chunk = blockIdx.x % a.cpp;
  const int G = gridDim.x / a.cpp;
  const int g = blockIdx.x / a.cpp;
  const long long planes = (long long)a.nvx * a.nvy;
  const long long n_items = g < planes ? (planes - g + G - 1) / G : 0;
  const long long plane_elems = (long long)nx * ny;

  if (threadIdx.x == 0) {
    for (int st = 0; st < S; ++st) mbar_init(&bars[st], 1);
    mbar_fence_init();
  }
  stage_lines11<T>(a.tx, a.nvx, xrec);
  stage_lines11<T>(a.ty, a.nvy, yrec);
  __syncthreads();

  auto issue = [&](long long it) {
    const long long p = g + it * G;
    int phys = (chunk * R + yrec[(int)(p / a.nvx)].m) % ny;
    uint64_t *bar = &bars[it % S];
    mbar_arrive_expect_tx(bar, slot_bytes);
    const T *src = static_cast<const T *>(a.fin) + p * plane_elems;
    T *dst = slots + (size_t)(it % S) * slot_elems;
    int remaining = vrows;
    while (remaining > 0) {
      const int len = remaining < ny - phys ? remaining : ny - phys;
      bulk_load(dst, src + (long long)phys * nx, (uint32_t)((size_t)len * nx * sizeof(T)), bar);
      dst += (size_t)len * nx;
      remaining -= len;
      phys = 0;
    }
  };
  if (threadIdx.x == 0) {
    const long long pre = n_items < S ? n_items : S;
    for (long long it = 0; it < pre; ++it) issue(it);
  }

  double racc[RT][4];
#pragma unroll
  for (int i = 0; i < RT; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) racc[i][q] = 0.0;

  // Trip count of the warp's first row group in the X11 phase, so that every
  // lane reaches each __syncwarp; the lanes this warp has.
  const int rgw = (int)((threadIdx.x & ~31u) / (unsigned)ncg);
  const int trips = (vrows - rgw + RG - 1) / RG;
  const unsigned wl = blockDim.x - (threadIdx.x & ~31u);
  const unsigned wmask = wl >= 32 ? 0xffffffffu : (1u << wl) - 1u;

  const int gdx = G % a.nvx, gdy = G / a.nvx;
  int ivx = g % a.nvx, ivy = g / a.nvx;
  int slot = 0;
  uint32_t parity = 0;
  for (long long it = 0; it < n_items; ++it) {
    const bool ok = mbar_wait_bounded(&bars[slot], parity);
    const long long p = g + it * G;
    T *in = slots + (size_t)slot * slot_elems;
    T *outp = static_cast<T *>(a.fout) + p * plane_elems + (long long)chunk * R * nx;
    {  // X11 in place on the staged rows rg, rg + RG, ... (this warp's rows),
       // output pairs at columns yc and yc + nx/2 (16-byte accesses,
       // consecutive across the lanes).
      W11<T> wx;
      int ba = (yc + read_line11(xrec[ivx], wx)) % nx;  // first tap of the pair at yc
      const int rr = ba & 1;                            // the same for both pairs (nx/2 is even)
      ba -= rr;
      const int bb = ba + nx / 2 >= nx ? ba - nx / 2 : ba + nx / 2;
      for (int k = 0; k < trips; ++k) {
        const int v = rg + k * RG;
        T *row = in + (size_t)v * nx;
        T outa[2], outb[2];
        if (v < vrows) {
          x11_pair_row(row, ba, nx, rr, wx, outa);
          x11_pair_row(row, bb, nx, rr, wx, outb);
        }
        __syncwarp(wmask);  // every lane has read the row
        if (v < vrows) {
          *reinterpret_cast<double2 *>(row + yc) = make_double2(outa[0], outa[1]);
          *reinterpret_cast<double2 *>(row + yc + nx / 2) = make_double2(outb[0], outb[1]);
        }
      }
      // These generic writes precede the slot's next bulk copy.
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    // The x-swept rows are complete; every thread is done with item it - 1,
    // whose slot now takes item it - 1 + S.
    const long long issued_end = it == 0 ? (long long)S : it - 1 + S;
    if (__syncthreads_or(!ok)) {
      plane_abort(a, bars, it, n_items, S, issued_end);
      return;
    }
    if (threadIdx.x == 0 && it > 0 && it - 1 + S < n_items) issue(it - 1 + S);
    {  // Y11 of rows r0 .. r0+RT-1, columns yc, yc+1, yc+nx/2, yc+nx/2+1,
       // streamed down the slot (16-byte accesses, consecutive across the
       // lanes: no bank conflicts).
      W11<T> wy;
      read_line11(yrec[ivy], wy);
      const T *src = in + (size_t)r0 * nx + yc;
      T acc[RT][4];
#pragma unroll
      for (int j = 0; j < RT + 10; ++j) {
        T y[4];
        {
          const double2 lo = *reinterpret_cast<const double2 *>(src + (size_t)j * nx);
          const double2 hi = *reinterpret_cast<const double2 *>(src + (size_t)j * nx + nx / 2);
          y[0] = lo.x;
          y[1] = lo.y;
          y[2] = hi.x;
          y[3] = hi.y;
        }
#pragma unroll
        for (int i = 0; i < RT; ++i) {
          const int k = j - i;
          if (k < 0 || k > 10) continue;
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[i][q] = k == 0 ? wy.w[0] * y[q] : fma(wy.w[k], y[q], acc[i][q]);
        }
        if (j >= 10) {
          const int i = j - 10;
          T *orow = outp + (size_t)(r0 + i) * nx + yc;
          *reinterpret_cast<double2 *>(orow) = make_double2(acc[i][0], acc[i][1]);
          *reinterpret_cast<double2 *>(orow + nx / 2) = make_double2(acc[i][2], acc[i][3]);
          if constexpr (RHO) {
#pragma unroll
            for (int q = 0; q < 4; ++q) racc[i][q] += acc[i][q];
          }
        }
      }
    }
    ivx += gdx;
    ivy += gdy;
    if (ivx >= a.nvx) {
      ivx -= a.nvx;
      ++ivy;
    }
    if (++slot == S) {
      slot = 0;
      parity ^= 1u;
    }
  }
  if constexpr (RHO) {
    double *rdst = a.rho_part + (long long)g * plane_elems + ((long long)chunk * R + r0) * nx + yc;
#pragma unroll
    for (int i = 0; i < RT; ++i) {
      *reinterpret_cast<double2 *>(rdst + (size_t)i * nx) = make_double2(racc[i][0], racc[i][1]);
      *reinterpret_cast<double2 *>(rdst + (size_t)i * nx + nx / 2) = make_double2(racc[i][2], racc[i][3]);
    }
  }
}

}  // namespace
}  // namespace vlp4d

namespace vlp4d {

namespace {

struct PlaneCfg {
  int R = 0, rt = 1, stages = 3, threads = 0, cpp = 1, grid = 0, G = 0;
  size_t smem = 0;
  int per_sm = 0;
  bool inplace = false;
};

int env_int(const char *name, int dflt) {
  const char *v = getenv(name);
  return v && *v ? atoi(v) : dflt;
}

size_t plane_smem(int R, int halo, int nx, size_t elem, int stages, bool dx, bool dy, int nvx, int nvy,
                  bool inplace = false) {
  const size_t slot = (size_t)(R + halo) * nx * elem;
  const size_t rec = elem == 4 ? 32 : 64;
  return kBarBytes + rec * ((dx ? nvx : 0) + (dy ? nvy : 0)) + stages * slot + ((dx && dy && !inplace) ? 2 * slot : 0);
}

// Chooses the chunk height R, rows per thread RT, the pipeline depth and the
// block size nx/4 * R/RT.  R is the tallest divisor of ny up to 32, 64 for
// the in-place FP64 x+y form (the halo re-read is 5/R of the rows, served
// from L2); then the deepest pipeline (3, else 2 stages) that lets
// two CTAs share an SM, else one CTA per SM with 3 stages.
// VLP4D_PLANE_R / _STAGES / _RT override for tuning sweeps.
bool plane_config(const vlp4d_ctx *c, bool dx, bool dy, PlaneCfg &cfg) {
  const int nx = c->g.n[0], ny = c->g.n[1];
  const size_t elem = c->elem;
  if (nx % 4 != 0 || nx > 2048) return false;
  const int halo = dy ? 5 : 0;
  const int ncg = nx / 4;
  const int forced_r = env_int("VLP4D_PLANE_R", 0);
  const int forced_rt = env_int("VLP4D_PLANE_RT", 0);
  const int forced_s = env_int("VLP4D_PLANE_STAGES", 0);
  // FP64 x+y: x-swept rows in place (no separate tiles) when a warp holds
  // whole rows; VLP4D_PLANE_INPLACE=0 turns it off.
  const bool inplace = elem == 8 && dx && dy && 32 % ncg == 0 && env_int("VLP4D_PLANE_INPLACE", 1) != 0;
  // Chunks of up to 32 rows; up to 64 for the in-place FP64 form, whose x
  // sweep also covers the five halo rows (7.8% extra at 64 rows, 15.6% at
  // 32): at 128^4, 64 rows in three stages (one 512-thread CTA per SM)
  // measured 0.768 against 0.844 ms; FP32 x+y was slower with 64 (0.430
  // against 0.412 ms).
  int R = 0, rt = 1;
  const int rmax = forced_r > 32 ? forced_r : (inplace ? 64 : 32);
  for (int r = ny < rmax ? ny : rmax; r >= 1; --r) {
    if (ny % r) continue;
    if (forced_r && r != forced_r) continue;
    const int t = forced_rt ? forced_rt : (r % 4 == 0 ? 4 : 1);
    if (t != 1 && t != 4 && t != 8) continue;
    if (r % t || ncg * (r / t) > 512) continue;
    R = r;
    rt = t;
    break;
  }
  if (!R) return false;
  const size_t two_per_sm = 112 * 1024, one_per_sm = 224 * 1024;
  int stages = 0;
  if (forced_s) {
    stages = forced_s;
  } else {
    for (int st = 3; st >= 2 && !stages; --st)
      if (plane_smem(R, halo, nx, elem, st, dx, dy, c->g.n[2], c->g.n[3], inplace) <= two_per_sm) stages = st;
    if (!stages) stages = 3;
  }
  if (stages < 2 || stages > kMaxStages) return false;
  const size_t smem = plane_smem(R, halo, nx, elem, stages, dx, dy, c->g.n[2], c->g.n[3], inplace);
  if (smem > one_per_sm) return false;
  cfg.R = R;
  cfg.rt = rt;
  cfg.stages = stages;
  cfg.cpp = ny / R;
  cfg.threads = ncg * (R / rt);
  cfg.smem = smem;
  cfg.inplace = inplace;
  return true;
}

// Widths whose rows a warp holds whole (nx/4 divides 32), or the run-time width.
constexpr bool inplace_width(int nx) { return nx == 0 || (nx % 4 == 0 && nx / 4 <= 32 && 32 % (nx / 4) == 0); }

template <typename T, int NX, int RT, bool DX, bool DY, bool RHO>
int run_plane(vlp4d_ctx *c, const PlaneArgs &args, PlaneCfg &cfg, cudaStream_t s) {
  auto kern = k_plane<T, NX, RT, DX, DY, RHO>;
  if constexpr (sizeof(T) == 8 && DX && DY && inplace_width(NX)) {
    if (cfg.inplace) kern = k_plane<T, NX, RT, DX, DY, RHO, true>;
  }
  VLP4D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem));
  int per_sm = 0;
  VLP4D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, cfg.threads, cfg.smem));
  if (per_sm < 1) return VLP4D_ERR_UNSUPPORTED;
  cfg.per_sm = per_sm;
  const long long planes = (long long)args.nvx * args.nvy;
  long long G = ((long long)per_sm * c->num_sms) / cfg.cpp;
  if (G < 1) G = 1;
  if (G > planes) G = planes;
  if (RHO && G > c->rho_part_groups) G = c->rho_part_groups;
  cfg.G = (int)G;
  cfg.grid = (int)G * cfg.cpp;
  kern<<<cfg.grid, cfg.threads, cfg.smem, s>>>(args);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

// Row-width specialisations: the common power-of-two widths get a
// compile-time nx (index math folds, wraps become masks), others run with
// the width read at run time.
template <typename T, int RT, bool DX, bool DY, bool RHO>
int run_plane_nx(vlp4d_ctx *c, const PlaneArgs &args, PlaneCfg &cfg, cudaStream_t s) {
  switch (args.nx) {
    case 64: return run_plane<T, 64, RT, DX, DY, RHO>(c, args, cfg, s);
    case 128: return run_plane<T, 128, RT, DX, DY, RHO>(c, args, cfg, s);
    case 256: return run_plane<T, 256, RT, DX, DY, RHO>(c, args, cfg, s);
    default: return run_plane<T, 0, RT, DX, DY, RHO>(c, args, cfg, s);
  }
}

template <typename T, bool DX, bool DY, bool RHO>
int run_plane_rt(vlp4d_ctx *c, const PlaneArgs &args, PlaneCfg &cfg, cudaStream_t s) {
  if (cfg.rt == 8) return run_plane_nx<T, 8, DX, DY, RHO>(c, args, cfg, s);
  if (cfg.rt == 4) return run_plane_nx<T, 4, DX, DY, RHO>(c, args, cfg, s);
  return run_plane_nx<T, 1, DX, DY, RHO>(c, args, cfg, s);
}

}  // namespace

namespace {

PlaneArgs plane_args(const vlp4d_ctx *c, const void *fn, void *fnp1, const PlaneCfg &cfg, int halo) {
  PlaneArgs a;
  a.fin = fn;
  a.fout = fnp1;
  a.nx = c->g.n[0];
  a.ny = c->g.n[1];
  a.nvx = c->g.n[2];
  a.nvy = c->g.n[3];
  a.R = cfg.R;
  a.cpp = cfg.cpp;
  a.halo = halo;
  a.stages = cfg.stages;
  a.rho_part = c->rho_part;
  a.err = c->d_err;
  return a;
}

size_t xyxy_smem(int R, int nx, size_t elem, int stages, int nvx, int nvy) {
  const size_t rec = elem == 4 ? 48 : 96;
  return kBarBytes + rec * (nvx + nvy) + (size_t)stages * (R + 10) * nx * elem + 2 * (size_t)R * nx * elem;
}

// Chunk height (the tallest divisor of ny up to 32 rows whose block and
// shared memory fit), rows per thread (4 in FP32 when R allows, 1 in FP64)
// and pipeline depth (3 stages if two CTAs then share an SM, else 2) of
// k_plane_xyxy.  VLP4D_XYXY_STAGES overrides the depth, VLP4D_XYXY_R the
// chunk height (tuning sweeps).
bool xyxy_config(const vlp4d_ctx *c, PlaneCfg &cfg) {
  const int nx = c->g.n[0], ny = c->g.n[1];
  if (nx % 4 != 0 || nx > 2048) return false;
  const int ncg = nx / 4;
  const int forced = env_int("VLP4D_XYXY_STAGES", 0);
  const int forced_r = env_int("VLP4D_XYXY_R", 0);
  if (forced && (forced < 2 || forced > kMaxStages)) return false;
  cfg.R = 0;
  const int rmax = forced_r > 0 ? forced_r : 32;
  for (int r = ny < rmax ? ny : rmax; r >= 1 && !cfg.R; --r) {
    if (ny % r) continue;
    if (forced_r && r != forced_r) continue;
    const int t = (c->elem == 4 && r % 4 == 0) ? 4 : 1;
    if (ncg * (r / t) > 512 || ncg * (r / t) < 1) continue;
    int st = forced;
    if (!st) {
      st = xyxy_smem(r, nx, c->elem, 3, c->g.n[2], c->g.n[3]) <= 112 * 1024 ? 3 : 2;
    }
    if (xyxy_smem(r, nx, c->elem, st, c->g.n[2], c->g.n[3]) > 224 * 1024) continue;
    cfg.R = r;
    cfg.rt = t;
    cfg.stages = st;
  }
  if (!cfg.R) return false;
  cfg.cpp = ny / cfg.R;
  cfg.threads = ncg * (cfg.R / cfg.rt);
  cfg.smem = xyxy_smem(cfg.R, nx, c->elem, cfg.stages, c->g.n[2], c->g.n[3]);
  return true;
}

// The X8 mapping for FP32 (VLP4D_XYXY_X8 = 0 turns it off).
bool xyxy_x8(int nx) {
  static const int env = env_int("VLP4D_XYXY_X8", 1);
  return env != 0 && nx % 8 == 0;
}

template <typename T, int NX, int RT>
int run_xyxy(vlp4d_ctx *c, const PlaneArgs &args, PlaneCfg &cfg, bool rho, cudaStream_t s) {
  auto kern = k_plane_xyxy<T, NX, RT>;
  if constexpr (sizeof(T) == 4 && RT == 4) {
    if (xyxy_x8(args.nx)) kern = rho ? k_plane_xyxy<T, NX, RT, true> : k_plane_xyxy<T, NX, RT, true, false>;
  }
  VLP4D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem));
  int per_sm = 0;
  VLP4D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, cfg.threads, cfg.smem));
  if (per_sm < 1) return VLP4D_ERR_UNSUPPORTED;
  cfg.per_sm = per_sm;
  const long long planes = (long long)args.nvx * args.nvy;
  long long G = ((long long)per_sm * c->num_sms) / cfg.cpp;
  if (G < 1) G = 1;
  if (G > planes) G = planes;
  if (G > c->rho_part_groups) G = c->rho_part_groups;
  cfg.G = (int)G;
  cfg.grid = (int)G * cfg.cpp;
  kern<<<cfg.grid, cfg.threads, cfg.smem, s>>>(args);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

template <typename T, int RT>
int run_xyxy_nx(vlp4d_ctx *c, const PlaneArgs &args, PlaneCfg &cfg, bool rho, cudaStream_t s) {
  switch (args.nx) {
    case 64: return run_xyxy<T, 64, RT>(c, args, cfg, rho, s);
    case 128: return run_xyxy<T, 128, RT>(c, args, cfg, rho, s);
    case 256: return run_xyxy<T, 256, RT>(c, args, cfg, rho, s);
    default: return run_xyxy<T, 0, RT>(c, args, cfg, rho, s);
  }
}

// k_plane_xyxy64: FP64, row widths a warp holds whole.  Chunk height: the
// tallest divisor of ny up to 64 whose block fits, four rows per thread
// when it divides, else one (the X11 phase also sweeps the ten halo rows:
// 16% extra at 64 rows, 31% at 32; at 128^4, 64 rows and two stages in one
// 512-thread CTA per SM measured 1.050 against 1.080 ms for 32 rows in two
// CTAs); two stages (three when two CTAs per SM are out of reach anyway and
// three fit).  VLP4D_XYXY64=0 turns it off (the FP64 form of
// k_plane_xyxy then runs); VLP4D_XYXY_STAGES overrides the depth,
// VLP4D_XYXY64_R the chunk height.
size_t xyxy64_smem(int R, int nx, int stages, int nvx, int nvy) {
  return kBarBytes + sizeof(LineRec11<double>) * (size_t)(nvx + nvy) + (size_t)stages * (R + 10) * nx * 8;
}

}  // namespace

bool xyxy64_available(const vlp4d_ctx *c) {
  const int nx = c->g.n[0];
  return c->fused && c->dtype == VLP4D_F64 && nx % 4 == 0 && 32 % (nx / 4) == 0 && env_int("VLP4D_XYXY64", 1) != 0;
}

namespace {

bool xyxy64_config(const vlp4d_ctx *c, PlaneCfg &cfg) {
  const int nx = c->g.n[0], ny = c->g.n[1];
  if (c->dtype != VLP4D_F64 || nx % 4 != 0 || 32 % (nx / 4) != 0) return false;
  if (env_int("VLP4D_XYXY64", 1) == 0) return false;
  const int ncg = nx / 4;
  const int forced = env_int("VLP4D_XYXY_STAGES", 0);
  if (forced && (forced < 2 || forced > kMaxStages)) return false;
  const int forced_r = env_int("VLP4D_XYXY64_R", 0);  // chunk height, for tuning sweeps
  const int rmax = forced_r > 0 ? forced_r : 64;
  for (int r = ny < rmax ? ny : rmax; r >= 1; --r) {
    if (ny % r) continue;
    if (forced_r && r != forced_r) continue;
    const int t = r % 4 == 0 ? 4 : 1;
    const int threads = ncg * (r / t);
    if (threads > 512) continue;
    int st = forced ? forced : 2;
    if (!forced && xyxy64_smem(r, nx, 2, c->g.n[2], c->g.n[3]) > 112 * 1024 &&
        xyxy64_smem(r, nx, 3, c->g.n[2], c->g.n[3]) <= 224 * 1024)
      st = 3;
    const size_t smem = xyxy64_smem(r, nx, st, c->g.n[2], c->g.n[3]);
    if (smem > 224 * 1024) continue;
    cfg.R = r;
    cfg.rt = t;
    cfg.stages = st;
    cfg.cpp = ny / r;
    cfg.threads = threads;
    cfg.smem = smem;
    return true;
  }
  return false;
}

template <int NX, int RT>
int run_xyxy64(vlp4d_ctx *c, PlaneArgs args, PlaneCfg &cfg, bool rho, cudaStream_t s) {
  auto kern = rho ? k_plane_xyxy64<NX, RT, true> : k_plane_xyxy64<NX, RT, false>;
  VLP4D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem));
  int per_sm = 0;
  VLP4D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, cfg.threads, cfg.smem));
  if (per_sm < 1) return VLP4D_ERR_UNSUPPORTED;
  cfg.per_sm = per_sm;
  args.R = cfg.R;
  args.cpp = cfg.cpp;
  args.stages = cfg.stages;
  const long long planes = (long long)args.nvx * args.nvy;
  long long G = ((long long)per_sm * c->num_sms) / cfg.cpp;
  if (G < 1) G = 1;
  if (G > planes) G = planes;
  if (G > c->rho_part_groups) G = c->rho_part_groups;
  cfg.G = (int)G;
  cfg.grid = (int)G * cfg.cpp;
  kern<<<cfg.grid, cfg.threads, cfg.smem, s>>>(args);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

template <int RT>
int run_xyxy64_nx(vlp4d_ctx *c, const PlaneArgs &a, PlaneCfg &cfg, bool rho, cudaStream_t s) {
  switch (a.nx) {
    case 64: return run_xyxy64<64, RT>(c, a, cfg, rho, s);
    case 128: return run_xyxy64<128, RT>(c, a, cfg, rho, s);
    default: return run_xyxy64<0, RT>(c, a, cfg, rho, s);
  }
}

int run_xyxy_any(vlp4d_ctx *c, const PlaneArgs &a, PlaneCfg &cfg, bool rho, cudaStream_t s) {
  if (c->dtype == VLP4D_F64) {
    PlaneCfg c64;
    if (xyxy64_config(c, c64)) {
      const int rc = c64.rt == 4 ? run_xyxy64_nx<4>(c, a, c64, rho, s) : run_xyxy64_nx<1>(c, a, c64, rho, s);
      if (rc != VLP4D_ERR_UNSUPPORTED) {
        cfg = c64;
        return rc;
      }
    }
  }
  if (c->dtype == VLP4D_F64)
    return cfg.rt == 4 ? run_xyxy_nx<double, 4>(c, a, cfg, rho, s) : run_xyxy_nx<double, 1>(c, a, cfg, rho, s);
  return cfg.rt == 4 ? run_xyxy_nx<float, 4>(c, a, cfg, rho, s) : run_xyxy_nx<float, 1>(c, a, cfg, rho, s);
}


}  // namespace

// Returns VLP4D_ERR_UNSUPPORTED (without launching anything) when the shape
// or the buffers do not meet the kernel's requirements; the caller then
// uses the generic kernels.
int launch_advect_xy(vlp4d_ctx *c, const void *fn, void *fnp1, const StencilTable *tx, const StencilTable *ty,
                     bool do_x, bool do_y, bool with_rho, cudaStream_t s) {
  if (!c->fused) return VLP4D_ERR_UNSUPPORTED;
  if (((uintptr_t)fn & 15) || ((uintptr_t)fnp1 & 15)) return VLP4D_ERR_UNSUPPORTED;
  if (!do_x && !do_y) return VLP4D_ERR_UNSUPPORTED;
  PlaneCfg cfg;
  if (!plane_config(c, do_x, do_y, cfg)) return VLP4D_ERR_UNSUPPORTED;
  const bool moment = with_rho && do_x && do_y;
  PlaneArgs a = plane_args(c, fn, fnp1, cfg, do_y ? 5 : 0);
  if (tx) a.tx = *tx;
  if (ty) a.ty = *ty;
  int rc;
#define VLP4D_PLANE(T, DX, DY, RHO) rc = run_plane_rt<T, DX, DY, RHO>(c, a, cfg, s)
  if (c->dtype == VLP4D_F64) {
    if (do_x && do_y) { if (moment) VLP4D_PLANE(double, true, true, true); else VLP4D_PLANE(double, true, true, false); }
    else if (do_x) VLP4D_PLANE(double, true, false, false);
    else VLP4D_PLANE(double, false, true, false);
  } else {
    if (do_x && do_y) { if (moment) VLP4D_PLANE(float, true, true, true); else VLP4D_PLANE(float, true, true, false); }
    else if (do_x) VLP4D_PLANE(float, true, false, false);
    else VLP4D_PLANE(float, false, true, false);
  }
#undef VLP4D_PLANE
  if (rc) return rc;
  if (moment) return launch_rho_finish(c, cfg.G, s);
  if (with_rho) return launch_field_rho(c, fnp1, s);
  return VLP4D_OK;
}

// Two x/y half steps (the composed 11-tap stencils of tx, ty) and the
// moment of the result in one pass; returns VLP4D_ERR_UNSUPPORTED (nothing
// launched) when the shape does not fit.
int launch_advect_xyxy(vlp4d_ctx *c, const void *fn, void *fnp1, const StencilTable *tx, const StencilTable *ty,
                       cudaStream_t s) {
  if (!c->fused) return VLP4D_ERR_UNSUPPORTED;
  if (((uintptr_t)fn & 15) || ((uintptr_t)fnp1 & 15)) return VLP4D_ERR_UNSUPPORTED;
  PlaneCfg cfg;
  if (!xyxy_config(c, cfg)) return VLP4D_ERR_UNSUPPORTED;
  StencilTable *x11 = nullptr, *y11 = nullptr;
  int rc0;
  if ((rc0 = ensure_xy11_table(c, 0, tx->dt, &x11, s))) return rc0;
  if ((rc0 = ensure_xy11_table(c, 1, ty->dt, &y11, s))) return rc0;
  return launch_advect_xyxy_tables(c, fn, fnp1, x11, y11, true, s);
}

int launch_advect_xyxy_tables(vlp4d_ctx *c, const void *fn, void *fnp1, const StencilTable *x11,
                              const StencilTable *y11, bool with_rho, cudaStream_t s) {
  if (!c->fused) return VLP4D_ERR_UNSUPPORTED;
  if (((uintptr_t)fn & 15) || ((uintptr_t)fnp1 & 15)) return VLP4D_ERR_UNSUPPORTED;
  PlaneCfg cfg;
  if (!xyxy_config(c, cfg)) return VLP4D_ERR_UNSUPPORTED;
  PlaneArgs a = plane_args(c, fn, fnp1, cfg, 10);
  a.tx = *x11;
  a.ty = *y11;
  int rc = run_xyxy_any(c, a, cfg, with_rho, s);
  if (rc || !with_rho) return rc;
  return launch_rho_finish(c, cfg.G, s);
}

}  // namespace vlp4d
