// Batched ensemble: many independent vlp4d runs of uneven grids advanced in
// ONE persistent kernel launch (captured in a CUDA graph together with the
// initial condition and the scheduler reset).
//
// No reference counterpart: the reference runs one domain per process.  Each
// member is the single-process step of timestep.hpp:14-67 on its own grid,
// FP32 f with FP64 fields, with the Landau sum initial condition
// f0 = M(vx) M(vy) (1 + amp (cos kx + cos ky)).
//
// Work decomposition.  Member r's run is a sequence of stages
//   0: moment of f0                     tiles: nvy  (one vy row of planes each)
//   1: field solve, diagnostic 0        tiles: 1
//   per step t (stage 2 + 3t + sub):
//   sub 0: x, y (dt/2) + moment         tiles: ceil(nvy / rows) (rows vy rows each)
//          for t > 0 joined with the closing x, y (dt/2) of step t - 1
//          (no field solve separates them): x, y, x, y as the composed
//          11-tap stencils, as the single-run time loop does in FP32
//   sub 1: field solve, diagnostic t+1  tiles: 1
//   sub 2: vx, vy (dt)                  tiles: ceil(nx*ny / cc)   (cc columns each)
//   last:  x, y (dt/2), the closing half step of the last step   tiles: ceil(nvy / rows)
// A stage's tiles may start only when the member's previous stage is
// complete; different members are independent.  Scheduling is dynamic and
// wait-free: a CTA picks a member, atomically takes the next tile of the
// member's current stage (one 64-bit word per member holds (stage, next
// tile)), runs it and counts it done; the CTA that completes a stage's last
// tile advances the member's word to the next stage.  A CTA that finds no
// tile moves on to another member, so no CTA ever waits for a specific
// other CTA: progress does not depend on which CTAs are resident.  A CTA
// leaves when every member has finished, or (error flag set) when it has
// found no tile for about two seconds.
//
// Data written inside the kernel and read by other CTAs (f between stages,
// moment partials, fields) is read with L2-only loads (ld.global.cg): the
// SM-local L1 is not coherent across CTAs.  Visibility follows the counter
// chain: writers fence then count their tile done; the CTA that sees the
// stage complete fences before publishing the next stage; a CTA that takes
// a tile of the new stage fences before reading.
//
// The field solve of a member (nx, ny <= 64) is a 2D DFT in FP64 shared
// memory (direct sums with tabulated twiddles: a few hundred thousand
// multiply-adds), the spectral solve of efield.cpp:43-105 (kx0 = 2*pi/xmax,
// mode 0 zeroed), and the inverse DFT keeping the real part.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "internal.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace vlp4d {
namespace {

constexpr int kEnsMaxN = 64;  // largest nx, ny of a member (field solve in shared memory)

struct EnsRun {
  int n[4];
  double minp[4], maxp[4], dx[4];
  double dt, amp, k;
  long long f_off;  // element offset of f in the arenas (multiple of 64)
  long long p_off;  // moment partials: nvy * nx*ny doubles
  long long e_off;  // fields: ex, ey (2 * nx*ny doubles)
  long long d_off;  // diagnostic history: nsteps + 1 doubles
  long long l_off;  // line tables: nvx x lines then nvy y lines (dt/2 shifts)
  int rows;         // vy rows per tile of the x/y stages
};

// Default and largest idle limit of a CTA of k_ensemble: about two seconds
// at 1.9 GHz.
constexpr long long kEnsIdleLimit = 4000000000LL;

struct EnsLine;
struct EnsLine11;

struct EnsArgs {
  const EnsRun *runs;
  const EnsLine *lines;      // per member at l_off: x lines by ivx, y lines by ivy
  const EnsLine11 *lines11;  // the same lines composed with themselves (11 taps)
  int nruns, nsteps;
  float *F0, *F1;
  double *part, *fld, *nrj;
  unsigned long long *word;
  unsigned int *done;
  int *remaining;
  int *err;
  int cc;      // columns per vx/vy tile
  int maxnxy;  // largest nx*ny of a member (shared-memory layout)
  long long idle_limit;
};

// Stages of a run of nsteps steps (none but the moment and field solve of
// f0 when nsteps is 0).
__host__ __device__ __forceinline__ int total_stages_of(int nsteps) { return nsteps > 0 ? 3 + 3 * nsteps : 2; }

__device__ __forceinline__ int stage_tiles(const EnsRun &R, int S, int cc) {
  if (S == 0) return R.n[3];
  if (S == 1) return 1;
  const int sub = (S - 2) % 3;
  if (sub == 1) return 1;
  if (sub == 2) return (R.n[0] * R.n[1] + cc - 1) / cc;
  return (R.n[3] + R.rows - 1) / R.rows;  // sub 0 and the closing x, y stage
}

// Stencil record of one line: FP32 difference weights and the tap offset.
struct EnsLine {
  float v[6];
  int m;
};

__device__ __forceinline__ EnsLine ens_line(double disp, double hmin, double hmax, int n) {
  const LineStencil s = line_stencil(disp, hmin, hmax, n);
  EnsLine l;
  weights_to_f32(s.w, l.v);
  l.m = s.m;
  return l;
}

// 16-byte asynchronous global-to-shared copies (L2 only), in commit groups.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Shared memory of the plane stages: the moment (FP64, maxnxy cells), a ring
// of kEnsRing raw plane groups, the x-swept group, the x lines of the row.
constexpr int kEnsGroupCells = 4608;  // cells of one plane group (18 KB FP32)
constexpr int kEnsRing = 3;           // raw group buffers: two groups in flight

// a / n for 0 <= a < 2^22, n >= 1, inv = 1.f / n: the float quotient is
// within one of the integer one, and one correction step fixes it.
__device__ __forceinline__ int div_small(int a, int n, float inv) {
  int q = __float2int_rz((float)a * inv);
  const int r = a - q * n;
  q += r >= n ? 1 : 0;
  q -= r < 0 ? 1 : 0;
  return q;
}

// Moment of f0 (stage 0) of the vy row `ivy`: the per-cell sum over the
// row's nvx planes in ivx order, FP64, to the row's partial.
__device__ void ens_moment0(const EnsArgs &a, const EnsRun &R, const float *fin, int ivy) {
  const int nvx = R.n[2];
  const int nxy = R.n[0] * R.n[1];
  const long long row0 = R.f_off + (long long)ivy * nvx * nxy;
  double *pp = a.part + R.p_off + (long long)ivy * nxy;
  for (int q = threadIdx.x; q < nxy; q += blockDim.x) {
    double s = 0.;
    for (int p = 0; p < nvx; ++p) s += (double)__ldcg(fin + row0 + (long long)p * nxy + q);
    pp[q] = s;
  }
}

// Composed 11-tap line of two shifts by the same displacement (the closing
// x/y half step of one step and the opening one of the next): out[i] =
// sum_q W_q in[(i + 2m + q) mod n], W = w * w, as FP32 difference weights
// about tap 5: out = f5 + sum_j u_j (f_{j+1} - f_j), u_j = -(W_0+..+W_j)
// for j < 5 and W_{j+1}+..+W_10 for j >= 5 (the weights sum to one).  FP64
// products and sums in the order of the single-run table, unfused.
struct EnsLine11 {
  float u[10];
  int m;
};

__device__ __forceinline__ EnsLine11 ens_line11(double disp, double hmin, double hmax, int n) {
  const LineStencil s = line_stencil(disp, hmin, hmax, n);
  double W[11];
#pragma unroll
  for (int q = 0; q < 11; ++q) W[q] = 0.;
#pragma unroll
  for (int k = 0; k < 6; ++k)
#pragma unroll
    for (int j = 0; j < 6; ++j) W[k + j] = __dadd_rn(W[k + j], __dmul_rn(s.w[k], s.w[j]));
  EnsLine11 l;
  double acc = 0.;
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    acc = __dadd_rn(acc, W[j]);
    l.u[j] = (float)-acc;
  }
  acc = 0.;
#pragma unroll
  for (int j = 9; j >= 5; --j) {
    acc = __dadd_rn(acc, W[j + 1]);
    l.u[j] = (float)acc;
  }
  l.m = (int)((2LL * s.m) % n);
  return l;
}

// f5 + sum_j u_j d_j on packed pairs.
__device__ __forceinline__ float2 ens_interp11(const float2 (&u)[10], float2 f5, const float2 *d) {
  float2 acc = __fmul2_rn(u[0], d[0]);
#pragma unroll
  for (int j = 1; j < 10; ++j) acc = __ffma2_rn(u[j], d[j], acc);
  return __fadd2_rn(f5, acc);
}

// Four X11 outputs from t[0..19] starting at the aligned column base - r:
// output q uses t[r+q .. r+q+10].
template <int R_>
__device__ __forceinline__ void ens_x11_from(const float (&t)[20], const float2 (&u)[10], float (&o)[4]) {
  float d[13];
#pragma unroll
  for (int j = 0; j < 13; ++j) d[j] = t[R_ + j + 1] - t[R_ + j];
  float2 dp[12];
#pragma unroll
  for (int j = 0; j < 12; ++j) dp[j] = make_float2(d[j], d[j + 1]);
  const float2 lo = ens_interp11(u, make_float2(t[R_ + 5], t[R_ + 6]), dp);
  const float2 hi = ens_interp11(u, make_float2(t[R_ + 7], t[R_ + 8]), dp + 2);
  o[0] = lo.x;
  o[1] = lo.y;
  o[2] = hi.x;
  o[3] = hi.y;
}

// One scalar output f5 + sum_j u_j (f_{j+1} - f_j).
__device__ __forceinline__ float ens_interp11_1(const float (&u)[10], const float (&t)[11]) {
  float acc = u[0] * (t[1] - t[0]);
#pragma unroll
  for (int j = 1; j < 10; ++j) acc = fmaf(u[j], t[j + 1] - t[j], acc);
  return t[5] + acc;
}

template <bool J11>
struct EnsLineOf {
  using T = EnsLine;
};
template <>
struct EnsLineOf<true> {
  using T = EnsLine11;
};

// x/y sweeps of the vy rows [tile * R.rows, tile * R.rows + R.rows) of
// member R.  MODE 0: x, y (dt/2); 1: x, y (dt/2) + moment; 2: x, y, x, y
// (dt/2 each) + moment, as the composed 11-tap stencils X11 then Y11 (the x
// and y shifts commute).  The tile's rows are contiguous in f (nvx planes of
// nx*ny cells each); each row is cut into groups of P planes (P * nx*ny <=
// kEnsGroupCells) and the tile's groups, row after row, stream through a
// ring of kEnsRing shared buffers with cp.async: two groups in flight while
// one is swept, across row boundaries, so that small members pay the ring's
// start-up once per tile of several rows.  Per group: the x sweep into the
// swept buffer, one barrier, the y sweep to global memory (items: every
// (plane, column quad) of the group, or two rows of a column quad in the
// joined form, so that small planes keep all threads busy).  With the
// moment the y sweep also leaves its output in the group's raw buffer (no
// longer read after the barrier), and after a second barrier the thread
// that owns cell q adds the group's planes to the cell's FP64 sum in ivx
// order, storing the row's sum after the row's last group: the sums do not
// depend on the block size or the tile configuration.  The lines come from
// the member's tables (x by ivx, y by ivy), built when the ensemble is
// created.
template <int MODE>
__device__ void ens_rows(const EnsArgs &a, const EnsRun &R, const float *fin, float *fout, int tile,
                         unsigned char *smem) {
  constexpr bool MOMENT = MODE >= 1;
  constexpr bool J11 = MODE == 2;
  using Line = typename EnsLineOf<J11>::T;
  const int nx = R.n[0], ny = R.n[1], nvx = R.n[2], nvy = R.n[3];
  const int nxy = nx * ny;
  const int y0 = tile * R.rows;
  const int nrows = nvy - y0 < R.rows ? nvy - y0 : R.rows;
  double *acc = reinterpret_cast<double *>(smem);
  float *raw0 = reinterpret_cast<float *>(acc + a.maxnxy);
  float *b1 = raw0 + (size_t)kEnsRing * kEnsGroupCells;
  Line *xl = reinterpret_cast<Line *>(b1 + kEnsGroupCells);
  const Line *tab;
  if constexpr (J11) tab = a.lines11 + R.l_off;
  else tab = a.lines + R.l_off;
  int P = kEnsGroupCells / nxy;
  P = P < 1 ? 1 : (P > nvx ? nvx : P);
  const int gpr = (nvx + P - 1) / P;  // groups per row
  const int ngroups = nrows * gpr;
  const long long tile0 = R.f_off + (long long)y0 * nvx * nxy;
  // Column quads when the rows are multiples of four floats (f_off is a
  // multiple of 64 elements, so every plane starts 16-byte aligned).
  const bool quad = (nx & 3) == 0;
  auto load_group = [&](int gi) {
    if (gi < ngroups) {
      const int r = gi / gpr;
      const int p0 = (gi - r * gpr) * P;
      const int np = nvx - p0 < P ? nvx - p0 : P;
      float *dst = raw0 + (size_t)(gi % kEnsRing) * kEnsGroupCells;
      const long long gbase = tile0 + ((long long)r * nvx + p0) * nxy;
      if (quad) {
        const float4 *src = reinterpret_cast<const float4 *>(fin + gbase);
        float4 *d4 = reinterpret_cast<float4 *>(dst);
        for (int c = threadIdx.x; c < (np * nxy) >> 2; c += blockDim.x) cp_async16(d4 + c, src + c);
      } else {
        for (int c = threadIdx.x; c < np * nxy; c += blockDim.x) dst[c] = __ldcg(fin + gbase + c);
      }
    }
    cp_async_commit();
  };
  // The ring's first loads go out before anything else; the previous tile
  // of this CTA has finished with every buffer (the scheduler's barrier).
#pragma unroll
  for (int gi = 0; gi < kEnsRing - 1; ++gi) load_group(gi);
  for (int l = threadIdx.x; l < nvx; l += blockDim.x) xl[l] = tab[l];
  if (MOMENT)
    for (int q = threadIdx.x; q < nxy; q += blockDim.x) acc[q] = 0.;
  for (int gi = 0; gi < ngroups; ++gi) {
    cp_async_wait<kEnsRing - 2>();
    // Group gi has landed (every thread's copies); every thread is done
    // with group gi - 1, whose buffer the next load reuses (at gi = 0: the
    // x lines are in place).
    __syncthreads();
    load_group(gi + kEnsRing - 1);
    const int r = gi / gpr;
    const int p0 = (gi - r * gpr) * P;
    const int np = nvx - p0 < P ? nvx - p0 : P;
    float *b0 = raw0 + (size_t)(gi % kEnsRing) * kEnsGroupCells;
    const long long gbase = tile0 + ((long long)r * nvx + p0) * nxy;
    const Line ly = tab[nvx + y0 + r];
    const int my = ly.m;
    if constexpr (!J11) {
      if (quad) {
        const int nq = nx >> 2, nqp = nxy >> 2;
        const float inv_nq = 1.f / (float)nq, inv_nqp = 1.f / (float)nqp;
        const int items = np * nqp;
        for (int it = threadIdx.x; it < items; it += blockDim.x) {
          const int p = div_small(it, nqp, inv_nqp);
          const int qi = it - p * nqp;
          const int iy = div_small(qi, nq, inv_nq);
          const int ix0 = (qi - iy * nq) << 2;
          const int row = p * nxy + iy * nx;
          const EnsLine &lx = xl[p0 + p];
          int base = ix0 + lx.m;
          base = base >= nx ? base - nx : base;
          const int rr = base & 3;
          int o[3];
          o[0] = base - rr;
          o[1] = o[0] + 4 >= nx ? o[0] + 4 - nx : o[0] + 4;
          o[2] = o[1] + 4 >= nx ? o[1] + 4 - nx : o[1] + 4;
          float t[12];
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const float4 v = *reinterpret_cast<const float4 *>(b0 + row + o[k]);
            t[4 * k] = v.x;
            t[4 * k + 1] = v.y;
            t[4 * k + 2] = v.z;
            t[4 * k + 3] = v.w;
          }
          SweepW<float> w;
          make_sweep_w(lx.v, w);
          float out[4];
          sweep_x4(t, rr, w, out);
          *reinterpret_cast<float4 *>(b1 + row + ix0) = make_float4(out[0], out[1], out[2], out[3]);
        }
        __syncthreads();
        SweepW<float> wy;
        make_sweep_w(ly.v, wy);
        for (int it = threadIdx.x; it < items; it += blockDim.x) {
          const int p = div_small(it, nqp, inv_nqp);
          const int qi = it - p * nqp;
          const int iy = div_small(qi, nq, inv_nq);
          const int ix0 = (qi - iy * nq) << 2;
          const float *pl = b1 + p * nxy + ix0;
          int j = iy + my;
          j = j >= ny ? j - ny : j;
          float2 y[6][2];
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            const float4 v = *reinterpret_cast<const float4 *>(pl + j * nx);
            y[k][0] = make_float2(v.x, v.y);
            y[k][1] = make_float2(v.z, v.w);
            if (++j == ny) j = 0;
          }
          float2 o2[2];
#pragma unroll
          for (int h = 0; h < 2; ++h)
            o2[h] = interp_diff2(wy.v, y[2][h], sub2(y[1][h], y[0][h]), sub2(y[2][h], y[1][h]), sub2(y[3][h], y[2][h]),
                                 sub2(y[4][h], y[3][h]), sub2(y[5][h], y[4][h]));
          const float4 o4 = make_float4(o2[0].x, o2[0].y, o2[1].x, o2[1].y);
          *reinterpret_cast<float4 *>(fout + gbase + (long long)it * 4) = o4;
          if (MOMENT) *reinterpret_cast<float4 *>(b0 + it * 4) = o4;
        }
      } else {
        const float inv_nx = 1.f / (float)nx, inv_nxy = 1.f / (float)nxy;
        const int cells = np * nxy;
        for (int c = threadIdx.x; c < cells; c += blockDim.x) {
          const int p = div_small(c, nxy, inv_nxy);
          const int qc = c - p * nxy;
          const int ix = qc - div_small(qc, nx, inv_nx) * nx;
          const int row = c - ix;
          const EnsLine &lx = xl[p0 + p];
          int j = ix + lx.m;
          j = j >= nx ? j - nx : j;
          float t[6];
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            t[k] = b0[row + j];
            if (++j == nx) j = 0;
          }
          b1[c] = interp6(lx.v, t[0], t[1], t[2], t[3], t[4], t[5]);
        }
        __syncthreads();
        for (int c = threadIdx.x; c < cells; c += blockDim.x) {
          const int p = div_small(c, nxy, inv_nxy);
          const int qc = c - p * nxy;
          const int iy = div_small(qc, nx, inv_nx);
          const float *pl = b1 + p * nxy + (qc - iy * nx);
          int j = iy + my;
          j = j >= ny ? j - ny : j;
          float t[6];
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            t[k] = pl[j * nx];
            if (++j == ny) j = 0;
          }
          const float o = interp6(ly.v, t[0], t[1], t[2], t[3], t[4], t[5]);
          fout[gbase + c] = o;
          if (MOMENT) b0[c] = o;
        }
      }
    } else {
      float2 uy[10];
      float uys[10];
#pragma unroll
      for (int k = 0; k < 10; ++k) {
        uys[k] = ly.u[k];
        uy[k] = make_float2(uys[k], uys[k]);
      }
      if (quad) {
        const int nq = nx >> 2, nqp = nxy >> 2;
        const float inv_nq = 1.f / (float)nq, inv_nqp = 1.f / (float)nqp;
        const int items = np * nqp;
        for (int it = threadIdx.x; it < items; it += blockDim.x) {
          const int p = div_small(it, nqp, inv_nqp);
          const int qi = it - p * nqp;
          const int iy = div_small(qi, nq, inv_nq);
          const int ix0 = (qi - iy * nq) << 2;
          const int row = p * nxy + iy * nx;
          const EnsLine11 &lx = xl[p0 + p];
          int base = ix0 + lx.m;
          base = base >= nx ? base - nx : base;
          const int rr = base & 3;
          int o = base - rr;
          float t[20];
#pragma unroll
          for (int k = 0; k < 5; ++k) {
            const float4 v = *reinterpret_cast<const float4 *>(b0 + row + o);
            t[4 * k] = v.x;
            t[4 * k + 1] = v.y;
            t[4 * k + 2] = v.z;
            t[4 * k + 3] = v.w;
            o += 4;
            if (o >= nx) o -= nx;
          }
          float2 u[10];
#pragma unroll
          for (int k = 0; k < 10; ++k) u[k] = make_float2(lx.u[k], lx.u[k]);
          float out[4];
          switch (rr) {
            case 0: ens_x11_from<0>(t, u, out); break;
            case 1: ens_x11_from<1>(t, u, out); break;
            case 2: ens_x11_from<2>(t, u, out); break;
            default: ens_x11_from<3>(t, u, out); break;
          }
          *reinterpret_cast<float4 *>(b1 + row + ix0) = make_float4(out[0], out[1], out[2], out[3]);
        }
        __syncthreads();
        if ((ny & 1) == 0) {
          // Y11 of two rows per item (iy, iy + 1 of one column quad): twelve
          // row loads and eleven differences serve both outputs, each computed
          // exactly as by the one-row items below.
          const int nq2 = nqp >> 1;
          const float inv_nq2 = 1.f / (float)nq2;
          const int items2 = np * nq2;
          for (int it = threadIdx.x; it < items2; it += blockDim.x) {
            const int p = div_small(it, nq2, inv_nq2);
            const int qi = it - p * nq2;
            const int iyp = div_small(qi, nq, inv_nq);
            const int ix0 = (qi - iyp * nq) << 2;
            const int iy = 2 * iyp;
            const float *pl = b1 + p * nxy + ix0;
            int j = iy + my;
            j = j >= ny ? j - ny : j;
            float2 y[12][2];
#pragma unroll
            for (int k = 0; k < 12; ++k) {
              const float4 v = *reinterpret_cast<const float4 *>(pl + j * nx);
              y[k][0] = make_float2(v.x, v.y);
              y[k][1] = make_float2(v.z, v.w);
              if (++j == ny) j = 0;
            }
            float2 o2[2][2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              float2 d[11];
#pragma unroll
              for (int k = 0; k < 11; ++k) d[k] = sub2(y[k + 1][h], y[k][h]);
              o2[0][h] = ens_interp11(uy, y[5][h], d);
              o2[1][h] = ens_interp11(uy, y[6][h], d + 1);
            }
#pragma unroll
            for (int rw = 0; rw < 2; ++rw) {
              const int cell = p * nxy + (iy + rw) * nx + ix0;
              const float4 o4 = make_float4(o2[rw][0].x, o2[rw][0].y, o2[rw][1].x, o2[rw][1].y);
              *reinterpret_cast<float4 *>(fout + gbase + cell) = o4;
              *reinterpret_cast<float4 *>(b0 + cell) = o4;
            }
          }
        } else {
          for (int it = threadIdx.x; it < items; it += blockDim.x) {
            const int p = div_small(it, nqp, inv_nqp);
            const int qi = it - p * nqp;
            const int iy = div_small(qi, nq, inv_nq);
            const int ix0 = (qi - iy * nq) << 2;
            const float *pl = b1 + p * nxy + ix0;
            int j = iy + my;
            j = j >= ny ? j - ny : j;
            float2 y[11][2];
#pragma unroll
            for (int k = 0; k < 11; ++k) {
              const float4 v = *reinterpret_cast<const float4 *>(pl + j * nx);
              y[k][0] = make_float2(v.x, v.y);
              y[k][1] = make_float2(v.z, v.w);
              if (++j == ny) j = 0;
            }
            float2 o2[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              float2 d[10];
#pragma unroll
              for (int k = 0; k < 10; ++k) d[k] = sub2(y[k + 1][h], y[k][h]);
              o2[h] = ens_interp11(uy, y[5][h], d);
            }
            const float4 o4 = make_float4(o2[0].x, o2[0].y, o2[1].x, o2[1].y);
            *reinterpret_cast<float4 *>(fout + gbase + (long long)it * 4) = o4;
            *reinterpret_cast<float4 *>(b0 + it * 4) = o4;
          }
        }
      } else {
        const float inv_nx = 1.f / (float)nx, inv_nxy = 1.f / (float)nxy;
        const int cells = np * nxy;
        for (int c = threadIdx.x; c < cells; c += blockDim.x) {
          const int p = div_small(c, nxy, inv_nxy);
          const int qc = c - p * nxy;
          const int ix = qc - div_small(qc, nx, inv_nx) * nx;
          const int row = c - ix;
          const EnsLine11 &lx = xl[p0 + p];
          int j = ix + lx.m;
          j = j >= nx ? j - nx : j;
          float t[11], u[10];
#pragma unroll
          for (int k = 0; k < 11; ++k) {
            t[k] = b0[row + j];
            if (++j == nx) j = 0;
          }
#pragma unroll
          for (int k = 0; k < 10; ++k) u[k] = lx.u[k];
          b1[c] = ens_interp11_1(u, t);
        }
        __syncthreads();
        for (int c = threadIdx.x; c < cells; c += blockDim.x) {
          const int p = div_small(c, nxy, inv_nxy);
          const int qc = c - p * nxy;
          const int iy = div_small(qc, nx, inv_nx);
          const float *pl = b1 + p * nxy + (qc - iy * nx);
          int j = iy + my;
          j = j >= ny ? j - ny : j;
          float t[11];
#pragma unroll
          for (int k = 0; k < 11; ++k) {
            t[k] = pl[j * nx];
            if (++j == ny) j = 0;
          }
          const float o = ens_interp11_1(uys, t);
          fout[gbase + c] = o;
          b0[c] = o;
        }
      }
    }
    if (MOMENT) {
      __syncthreads();  // the group's outputs are in b0
      const bool last = p0 + np == nvx;
      double *pp = a.part + R.p_off + (long long)(y0 + r) * nxy;
      for (int q = threadIdx.x; q < nxy; q += blockDim.x) {
        double s = acc[q];
        for (int p = 0; p < np; ++p) s += (double)b0[p * nxy + q];
        if (last) {
          pp[q] = s;  // the row's sum; cell q's next row starts from zero
          acc[q] = 0.;
        } else {
          acc[q] = s;
        }
      }
    }
  }
  cp_async_wait<0>();
}

// vx then vy (dt) of the columns [tile*cc, tile*cc + cc).  Thread (col, g)
// handles the groups of V consecutive output vx rows g, g+G, ...; for each
// group it streams the vy rows from the column's vy offset (V+5 vx taps per
// row, shared by the V outputs), keeping six vx-swept rows in a ring, with
// the taps of the next D rows in flight.
template <int D>
__device__ void ens_vxvy(const EnsArgs &a, const EnsRun &R, const float *fin, float *fout, int tile) {
  static_assert(6 % D == 0, "the tap ring is indexed by the unrolled row");
  constexpr int V = 4;
  const int nx = R.n[0], ny = R.n[1], nvx = R.n[2], nvy = R.n[3];
  const int nxy = nx * ny;
  const int cc = a.cc;
  const int G = blockDim.x / cc;
  const int lc = threadIdx.x % cc, g = threadIdx.x / cc;
  const int col = tile * cc + lc;
  if (g >= G || col >= nxy) return;
  const double *ex = a.fld + R.e_off, *ey = ex + nxy;
  const EnsLine lx = ens_line(R.dt * __ldcg(ex + col), R.minp[2], R.maxp[2], nvx);
  const EnsLine ly = ens_line(R.dt * __ldcg(ey + col), R.minp[3], R.maxp[3], nvy);
  // Offsets within the member's f (< 64^4 elements) fit 32 bits.
  const int ystride = nxy * nvx;
  const float *src = fin + R.f_off + col;
  float *dst = fout + R.f_off + col;
  const int nrows = nvy + 5;
  for (int v0 = g * V; v0 < nvx; v0 += G * V) {
    int toff[V + 5];
    int j = v0 + lx.m;
    while (j >= nvx) j -= nvx;
#pragma unroll
    for (int k = 0; k < V + 5; ++k) {
      toff[k] = j * nxy;
      if (++j == nvx) j = 0;
    }
    float ring[6][V];
    float t[D][V + 5];
    int lrow = ly.m;  // the next vy row to load
#pragma unroll
    for (int d = 0; d < D; ++d) {
      if (d < nrows) {
        const float *pn = src + lrow * ystride;
#pragma unroll
        for (int k = 0; k < V + 5; ++k) t[d][k] = __ldcg(pn + toff[k]);
        if (++lrow == nvy) lrow = 0;
      }
    }
    for (int r0 = 0; r0 < nrows; r0 += 6) {
#pragma unroll
      for (int u = 0; u < 6; ++u) {
        const int r = r0 + u;
        if (r >= nrows) break;
        float(&cur)[V + 5] = t[u % D];
#pragma unroll
        for (int i = 0; i < V; ++i)
          ring[u][i] = interp6(lx.v, cur[i], cur[i + 1], cur[i + 2], cur[i + 3], cur[i + 4], cur[i + 5]);
        if (r + D < nrows) {
          const float *pn = src + lrow * ystride;
#pragma unroll
          for (int k = 0; k < V + 5; ++k) cur[k] = __ldcg(pn + toff[k]);
          if (++lrow == nvy) lrow = 0;
        }
        if (r >= 5) {
          float *orow = dst + (r - 5) * ystride;
#pragma unroll
          for (int i = 0; i < V; ++i) {
            if (v0 + i < nvx)
              orow[(v0 + i) * nxy] = interp6(ly.v, ring[(u + 1) % 6][i], ring[(u + 2) % 6][i], ring[(u + 3) % 6][i],
                                             ring[(u + 4) % 6][i], ring[(u + 5) % 6][i], ring[u][i]);
          }
        }
      }
    }
  }
}

// One 1D DFT pass over a (rows x len) complex array in shared memory:
// out[r][k] = sum_j in[r][j] * w^(sign k j), w = exp(2 pi i / len); strides
// select rows/columns.  tw[m] = (cos(2 pi m/len), sin(2 pi m/len)).
__device__ void ens_dft(const double2 *in, double2 *out, int rows, int len, int rstride, int estride,
                        const double2 *tw, double sign) {
  for (int o = threadIdx.x; o < rows * len; o += blockDim.x) {
    const int r = o / len, k = o % len;
    double sr = 0., si = 0.;
    int m = 0;
    for (int j = 0; j < len; ++j) {
      const double2 v = in[r * rstride + j * estride];
      const double2 w = tw[m];
      const double wi = sign * w.y;
      sr = fma(v.x, w.x, fma(-v.y, wi, sr));
      si = fma(v.x, wi, fma(v.y, w.x, si));
      m += k;
      if (m >= len) m -= len;
    }
    out[r * rstride + k * estride] = make_double2(sr, si);
  }
}

// Field solve of member R from its moment partials, diagnostic slot `iter`.
// Shared memory: two complex (maxnxy) arrays and the twiddles.
__device__ void ens_field(const EnsArgs &a, const EnsRun &R, int iter, unsigned char *smem) {
  const int nx = R.n[0], ny = R.n[1], nvy = R.n[3];
  const int nxy = nx * ny;
  double2 *H1 = reinterpret_cast<double2 *>(smem);
  double2 *H2 = H1 + a.maxnxy;
  double2 *twx = H2 + a.maxnxy;
  double2 *twy = twx + kEnsMaxN;
  for (int m = threadIdx.x; m < nx; m += blockDim.x) {
    double sn, cs;
    sincospi(2.0 * m / nx, &sn, &cs);
    twx[m] = make_double2(cs, sn);
  }
  for (int m = threadIdx.x; m < ny; m += blockDim.x) {
    double sn, cs;
    sincospi(2.0 * m / ny, &sn, &cs);
    twy[m] = make_double2(cs, sn);
  }
  // rho = dvx dvy * (sum of the vy rows' partials, fixed order), as complex.
  const double dvv = R.dx[2] * R.dx[3];
  const double *p = a.part + R.p_off;
  for (int c = threadIdx.x; c < nxy; c += blockDim.x) {
    double sum = 0.;
    for (int v = 0; v < nvy; ++v) sum += __ldcg(p + (long long)v * nxy + c);
    H1[c] = make_double2(sum * dvv, 0.);
  }
  __syncthreads();
  ens_dft(H1, H2, ny, nx, nx, 1, twx, -1.);  // along x, every row
  __syncthreads();
  ens_dft(H2, H1, nx, ny, 1, nx, twy, -1.);  // along y, every column: H1 = rho_hat
  __syncthreads();
  const double kx0 = 2 * M_PI / R.maxp[0], ky0 = 2 * M_PI / R.maxp[1];
  const double norm = 1.0 / ((double)nx * ny);
  for (int comp = 0; comp < 2; ++comp) {
    // H2 = inverse DFT along y of (-i k_comp / |k|^2 / (nx ny)) * rho_hat
    // (mode 0 zeroed), column by column.
    for (int o = threadIdx.x; o < nxy; o += blockDim.x) {
      const int ix = o % nx, y = o / nx;
      const double kx = (ix <= nx / 2 ? ix : ix - nx) * kx0;
      double sr = 0., si = 0.;
      int m = 0;
      for (int iy = 0; iy < ny; ++iy) {
        const double ky = (iy <= ny / 2 ? iy : iy - ny) * ky0;
        const double k2 = kx * kx + ky * ky;
        const double q = (ix == 0 && iy == 0) ? 0. : (comp == 0 ? kx : ky) / k2 * norm;
        const double2 h = H1[iy * nx + ix];
        const double vr = q * h.y, vi = -q * h.x;
        const double2 w = twy[m];
        sr = fma(vr, w.x, fma(-vi, w.y, sr));
        si = fma(vr, w.y, fma(vi, w.x, si));
        m += y;
        if (m >= ny) m -= ny;
      }
      H2[o] = make_double2(sr, si);
    }
    __syncthreads();
    // Real part of the inverse DFT along x, to the field arena.
    double *e = a.fld + R.e_off + (long long)comp * nxy;
    for (int o = threadIdx.x; o < nxy; o += blockDim.x) {
      const int x = o % nx, y = o / nx;
      double sr = 0.;
      int m = 0;
      for (int ix = 0; ix < nx; ++ix) {
        const double2 v = H2[y * nx + ix];
        const double2 w = twx[m];
        sr = fma(v.x, w.x, fma(-v.y, w.y, sr));
        m += x;
        if (m >= nx) m -= nx;
      }
      e[o] = sr;
    }
    __syncthreads();
  }
  // Energy: a fixed reduction order whatever the block size (lane l sums
  // cells l, l+32, ...; then a fixed shuffle tree), so the history does not
  // depend on the tile configuration.
  if (threadIdx.x < 32) {
    const double *ex = a.fld + R.e_off, *ey = ex + nxy;
    double e2 = 0.;
    for (int c = threadIdx.x; c < nxy; c += 32) e2 += ex[c] * ex[c] + ey[c] * ey[c];
    for (int o = 16; o > 0; o >>= 1) e2 += __shfl_down_sync(0xffffffffu, e2, o);
    if (threadIdx.x == 0) {
      const double en = sqrt(e2 * R.dx[0] * R.dx[1]);
      a.nrj[R.d_off + iter] = en > 1.e-30 ? log(en) : -1.e9;
    }
  }
}

__global__ void __launch_bounds__(512) k_ensemble(EnsArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_run, s_stage, s_tile;
  const int total_stages = total_stages_of(a.nsteps);
  // Scheduler state, kept (identically) by the lanes of warp 0.
  int r = (int)((blockIdx.x * 7919LL) % a.nruns);
  long long idle_start = clock64();
  const int lane = threadIdx.x & 31;
  while (true) {
    if (threadIdx.x < 32) {
      // Warp 0 looks for a tile: 32 members per round, starting at r (the
      // member last worked on), one sweep over all members at most.  Among
      // the members of a round with free tiles it tries the one with the
      // most work left first (stages left x cells), so that the largest
      // members do not finish alone at the end of the run.
      // got_run: -1 leave (all members done, or no work for idle_limit
      // cycles); -2 nothing taken; >= 0 a tile of that member.
      int got_run = -2, got_stage = 0, got_tile = 0;
      {
        const int rounds = (a.nruns + 31) / 32;
        for (int rd = 0; rd < rounds && got_run == -2; ++rd) {
          const int idx = rd * 32 + lane;
          const int cand = (int)(((long long)r + idx) % a.nruns);
          bool avail = false;
          unsigned key = 0;  // work left, 26 bits, at least 1 when avail
          if (idx < a.nruns) {
            const unsigned long long w = *(volatile unsigned long long *)(a.word + cand);
            const int stage = (int)(w >> 32);
            const EnsRun &Rc = a.runs[cand];
            avail = stage < total_stages && (int)(w & 0xffffffffu) < stage_tiles(Rc, stage, a.cc);
            if (avail) {
              const unsigned long long cells = (unsigned long long)Rc.n[0] * Rc.n[1] * Rc.n[2] * Rc.n[3];
              const unsigned long long work = (unsigned long long)(total_stages - stage) * ((cells >> 10) + 1);
              key = (unsigned)(work < (1ull << 26) - 1 ? work : (1ull << 26) - 2) + 1u;
            }
          }
          unsigned ballot = __ballot_sync(0xffffffffu, avail);
          while (ballot) {
            // Most work left first; lower lanes on ties.
            const unsigned mine = (ballot >> lane) & 1u ? (key << 5) | (31u - (unsigned)lane) : 0u;
            const int leader = 31 - (int)(__reduce_max_sync(0xffffffffu, mine) & 31u);
            int ok = 0, st = 0, tl = 0;
            if (lane == leader) {
              const unsigned long long got = atomicAdd(a.word + cand, 1ULL);
              st = (int)(got >> 32);
              tl = (int)(got & 0xffffffffu);
              ok = st < total_stages && tl < stage_tiles(a.runs[cand], st, a.cc);
              if (ok) __threadfence();
            }
            ok = __shfl_sync(0xffffffffu, ok, leader);
            if (ok) {
              got_run = __shfl_sync(0xffffffffu, cand, leader);
              got_stage = __shfl_sync(0xffffffffu, st, leader);
              got_tile = __shfl_sync(0xffffffffu, tl, leader);
              break;
            }
            ballot &= ~(1u << leader);
          }
        }
        if (got_run >= 0) {
          r = got_run;
          idle_start = clock64();
        } else if (__shfl_sync(0xffffffffu, lane == 0 ? *(volatile int *)a.remaining : 0, 0) <= 0) {
          got_run = -1;  // every member has finished
        } else {
          __nanosleep(256);
          if (clock64() - idle_start > a.idle_limit) {
            if (lane == 0) atomicExch(a.err, 1);
            got_run = -1;
          }
          got_run = __shfl_sync(0xffffffffu, got_run, 0);
        }
      }
      if (lane == 0) {
        s_run = got_run;
        s_stage = got_stage;
        s_tile = got_tile;
      }
    }
    __syncthreads();
    const int run = s_run;
    if (run == -1) break;
    if (run >= 0) {
      const EnsRun &R = a.runs[run];
      const int S = s_stage, tile = s_tile;
      if (S == 0) {
        ens_moment0(a, R, a.F0, tile);
      } else if (S == 1) {
        ens_field(a, R, 0, smem);
      } else if (S + 1 == total_stages) {
        ens_rows<0>(a, R, a.F0, a.F1, tile, smem);  // closing half step
      } else {
        // The state lives in F0 between steps; sub 0 writes F1, vx/vy F0.
        const int t = (S - 2) / 3, sub = (S - 2) % 3;
        if (sub == 0) {
          if (t == 0) ens_rows<1>(a, R, a.F0, a.F1, tile, smem);
          else ens_rows<2>(a, R, a.F0, a.F1, tile, smem);
        } else if (sub == 1) {
          ens_field(a, R, t + 1, smem);
        } else {
          ens_vxvy<3>(a, R, a.F1, a.F0, tile);
        }
      }
      // Every thread's writes, then the tile count.
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) {
        const unsigned int n = (unsigned int)stage_tiles(R, S, a.cc);
        if (atomicAdd(a.done + run, 1u) + 1u == n) {
          a.done[run] = 0u;
          __threadfence();
          if (S + 1 == total_stages) atomicSub(a.remaining, 1);
          atomicExch(a.word + run, (unsigned long long)(S + 1) << 32);
        }
      }
    }
    __syncthreads();
  }
}

__global__ void k_ens_init(EnsArgs a) {
  const EnsRun &R = a.runs[blockIdx.y];
  const long long total = (long long)R.n[0] * R.n[1] * R.n[2] * R.n[3];
  const double PI = 3.14159265358979323846;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(idx % R.n[0]);
    long long q = idx / R.n[0];
    const int iy = (int)(q % R.n[1]);
    q /= R.n[1];
    const int ivx = (int)(q % R.n[2]);
    const int ivy = (int)(q / R.n[2]);
    const double x = R.minp[0] + ix * R.dx[0];
    const double y = R.minp[1] + iy * R.dx[1];
    const double vx = R.minp[2] + ivx * R.dx[2];
    const double vy = R.minp[3] + ivy * R.dx[3];
    const double val = (1. + R.amp * cos(R.k * x) + R.amp * cos(R.k * y)) * (exp(-0.5 * (vx * vx + vy * vy)) / (2 * PI));
    a.F0[R.f_off + idx] = (float)val;
  }
}

// Line tables of every member (one block each): the dt/2 shifts of the x/y
// stages, x lines by ivx (displacement dt/2 * vx) and y lines by ivy
// (dt/2 * vy), as single lines and composed with themselves.  Built once
// per ensemble: they depend only on the member's grid and dt.
__global__ void k_ens_lines(const EnsRun *runs, EnsLine *lines, EnsLine11 *lines11) {
  const EnsRun &R = runs[blockIdx.x];
  const double hdt = 0.5 * R.dt;
  const int nx = R.n[0], ny = R.n[1], nvx = R.n[2], nvy = R.n[3];
  EnsLine *l1 = lines + R.l_off;
  EnsLine11 *l2 = lines11 + R.l_off;
  for (int l = threadIdx.x; l < nvx; l += blockDim.x) {
    const double disp = hdt * (R.minp[2] + l * R.dx[2]);
    l1[l] = ens_line(disp, R.minp[0], R.maxp[0], nx);
    l2[l] = ens_line11(disp, R.minp[0], R.maxp[0], nx);
  }
  for (int l = threadIdx.x; l < nvy; l += blockDim.x) {
    const double disp = hdt * (R.minp[3] + l * R.dx[3]);
    l1[nvx + l] = ens_line(disp, R.minp[1], R.maxp[1], ny);
    l2[nvx + l] = ens_line11(disp, R.minp[1], R.maxp[1], ny);
  }
}

__global__ void k_ens_reset(EnsArgs a) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < a.nruns) {
    a.word[r] = 0ull;
    a.done[r] = 0u;
  }
  if (r == 0) {
    *a.remaining = a.nruns;
    *a.err = 0;
  }
}

}  // namespace
}  // namespace vlp4d

struct vlp4d_ensemble {
  int device = 0, num_sms = 0;
  int nruns = 0, nsteps = 0;
  std::vector<vlp4d::EnsRun> host_runs;
  vlp4d::EnsRun *runs = nullptr;
  vlp4d::EnsLine *lines = nullptr;
  vlp4d::EnsLine11 *lines11 = nullptr;
  float *F[2] = {nullptr, nullptr};
  double *part = nullptr, *fld = nullptr, *nrj = nullptr;
  unsigned long long *word = nullptr;
  unsigned int *done = nullptr;
  int *remaining = nullptr, *err = nullptr;
  long long total_cells = 0, max_cells = 0;
  int maxnxy = 0;
  // Tile configuration (vlp4d_ensemble_set_tiles / _autotune).
  int threads = 256, cc = 32, ctas_per_sm = 0;  // 0: as many as fit
  size_t smem = 0;
  // Cycles a CTA may look for work in vain before it flags a timeout and
  // leaves (vlp4d_ensemble_set_idle_limit).
  long long idle_limit = vlp4d::kEnsIdleLimit;
  cudaGraphExec_t graph = nullptr;
};

namespace vlp4d {
namespace {

size_t ens_smem(int maxnxy) {
  const size_t line = sizeof(EnsLine11) > sizeof(EnsLine) ? sizeof(EnsLine11) : sizeof(EnsLine);
  const size_t planes = sizeof(double) * maxnxy + (kEnsRing + 1) * sizeof(float) * kEnsGroupCells + line * kEnsMaxN;
  const size_t field = 2 * sizeof(double2) * maxnxy + 2 * sizeof(double2) * kEnsMaxN;
  return ((planes > field ? planes : field) + 255) / 256 * 256;
}

EnsArgs ens_args(vlp4d_ensemble *E, int nsteps) {
  EnsArgs a;
  a.runs = E->runs;
  a.lines = E->lines;
  a.lines11 = E->lines11;
  a.nruns = E->nruns;
  a.nsteps = nsteps;
  a.F0 = E->F[0];
  a.F1 = E->F[1];
  a.part = E->part;
  a.fld = E->fld;
  a.nrj = E->nrj;
  a.word = E->word;
  a.done = E->done;
  a.remaining = E->remaining;
  a.err = E->err;
  a.cc = E->cc;
  a.maxnxy = E->maxnxy;
  a.idle_limit = E->idle_limit;
  return a;
}

// Initial condition, scheduler reset and the persistent launch.
int ens_launch(vlp4d_ensemble *E, int nsteps, cudaStream_t s) {
  const EnsArgs a = ens_args(E, nsteps);
  dim3 ig((unsigned)((E->max_cells + 255) / 256 < 4096 ? (E->max_cells + 255) / 256 : 4096), (unsigned)E->nruns);
  k_ens_init<<<ig, 256, 0, s>>>(a);
  VLP4D_LAUNCH_CHECK();
  k_ens_reset<<<(E->nruns + 255) / 256, 256, 0, s>>>(a);
  VLP4D_LAUNCH_CHECK();
  int per_sm = 0;
  VLP4D_CUDA_TRY(cudaFuncSetAttribute(k_ensemble, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)E->smem));
  VLP4D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ensemble, E->threads, E->smem));
  if (per_sm < 1) return fail_msg(VLP4D_ERR_UNSUPPORTED, "ensemble: tile configuration does not fit an SM");
  if (E->ctas_per_sm > 0 && E->ctas_per_sm < per_sm) per_sm = E->ctas_per_sm;
  k_ensemble<<<per_sm * E->num_sms, E->threads, E->smem, s>>>(a);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

void ens_free(vlp4d_ensemble *E) {
  if (!E) return;
  if (E->graph) cudaGraphExecDestroy(E->graph);
  cudaFree(E->runs);
  cudaFree(E->lines);
  cudaFree(E->lines11);
  cudaFree(E->F[0]);
  cudaFree(E->F[1]);
  cudaFree(E->part);
  cudaFree(E->fld);
  cudaFree(E->nrj);
  cudaFree(E->word);
  cudaFree(E->done);
  cudaFree(E->remaining);
  delete E;
}

int ens_check(vlp4d_ensemble *E) {
  int h = 0;
  VLP4D_CUDA_TRY(cudaMemcpy(&h, E->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) return fail_msg(VLP4D_ERR_TIMEOUT, "ensemble: a CTA found no work for its whole time limit");
  return VLP4D_OK;
}

// Makes the ensemble's device current for the duration of an API call and
// restores the caller's device afterwards, so that graph capture, launches
// and synchronisation always target the device the ensemble lives on.
struct EnsDeviceScope {
  int prev = -1;
  bool ok = false;
  explicit EnsDeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    ok = prev == dev || cudaSetDevice(dev) == cudaSuccess;
    if (!ok) cudaGetLastError();
  }
  ~EnsDeviceScope() {
    if (ok && prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace
}  // namespace vlp4d

using namespace vlp4d;

extern "C" {

int vlp4d_ensemble_create(const vlp4d_ens_member *members, int nruns, int nsteps, vlp4d_ensemble **out) {
  if (!out) return fail_msg(VLP4D_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (!members || nruns < 1) return fail_msg(VLP4D_ERR_INVALID_ARG, "no members");
  if (nsteps < 0 || nsteps > (1 << 28)) return fail_msg(VLP4D_ERR_INVALID_ARG, "nsteps out of range");
  int dev = 0, nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd < 1) {
    cudaGetLastError();
    return fail_msg(VLP4D_ERR_NO_DEVICE, "no CUDA device");
  }
  VLP4D_CUDA_TRY(cudaGetDevice(&dev));
  vlp4d_ensemble *E = new vlp4d_ensemble();
  E->device = dev;
  VLP4D_CUDA_TRY(cudaDeviceGetAttribute(&E->num_sms, cudaDevAttrMultiProcessorCount, dev));
  E->nruns = nruns;
  E->nsteps = nsteps;
  long long foff = 0, poff = 0, eoff = 0, doff = 0, loff = 0;
  // Cells per tile of the x/y stages: the vy rows of small members are
  // batched into tiles of about this many cells (one row at least), so that
  // the plane-group ring's start-up is paid once per tile.
  long long tile_cells = 131072;
  if (const char *env = getenv("VLP4D_ENS_TILE_CELLS")) tile_cells = atoll(env) > 0 ? atoll(env) : 1;
  for (int r = 0; r < nruns; ++r) {
    const vlp4d_ens_member &m = members[r];
    EnsRun R;
    for (int i = 0; i < 4; ++i) {
      if (m.n[i] < 1 || !(m.max_phy[i] > m.min_phy[i])) {
        ens_free(E);
        return fail_msg(VLP4D_ERR_INVALID_ARG, "ensemble member " + std::to_string(r) + ": bad extent or box");
      }
      R.n[i] = m.n[i];
      R.minp[i] = m.min_phy[i];
      R.maxp[i] = m.max_phy[i];
      R.dx[i] = (m.max_phy[i] - m.min_phy[i]) / m.n[i];
    }
    if (R.n[0] > kEnsMaxN || R.n[1] > kEnsMaxN || R.n[2] > kEnsMaxN) {
      ens_free(E);
      return fail_msg(VLP4D_ERR_UNSUPPORTED, "ensemble member " + std::to_string(r) + ": nx, ny, nvx must be at most 64");
    }
    if (!std::isfinite(m.dt)) {
      ens_free(E);
      return fail_msg(VLP4D_ERR_INVALID_ARG, "ensemble member " + std::to_string(r) + ": dt is not finite");
    }
    R.dt = m.dt;
    R.amp = m.amp;
    R.k = m.k;
    const long long nxy = (long long)R.n[0] * R.n[1];
    const long long cells = nxy * R.n[2] * R.n[3];
    R.f_off = foff;
    foff += (cells + 63) / 64 * 64;
    R.p_off = poff;
    poff += nxy * R.n[3];
    R.e_off = eoff;
    eoff += 2 * nxy;
    R.d_off = doff;
    doff += nsteps + 1;
    R.l_off = loff;
    loff += R.n[2] + R.n[3];
    {
      const long long row_cells = nxy * R.n[2];
      long long per = tile_cells / row_cells;
      per = per < 1 ? 1 : (per > R.n[3] ? R.n[3] : per);
      const long long tiles = (R.n[3] + per - 1) / per;
      R.rows = (int)((R.n[3] + tiles - 1) / tiles);  // balanced tiles
    }
    E->total_cells += cells;
    if (cells > E->max_cells) E->max_cells = cells;
    if (nxy > E->maxnxy) E->maxnxy = (int)nxy;
    E->host_runs.push_back(R);
  }
  E->maxnxy = (E->maxnxy + 3) / 4 * 4;  // 16-byte aligned shared-memory buffers
  E->smem = ens_smem(E->maxnxy);
  bool ok = cudaMalloc(&E->runs, sizeof(EnsRun) * nruns) == cudaSuccess &&
            cudaMalloc(&E->F[0], sizeof(float) * foff) == cudaSuccess &&
            cudaMalloc(&E->F[1], sizeof(float) * foff) == cudaSuccess &&
            cudaMalloc(&E->part, sizeof(double) * poff) == cudaSuccess &&
            cudaMalloc(&E->fld, sizeof(double) * eoff) == cudaSuccess &&
            cudaMalloc(&E->nrj, sizeof(double) * doff) == cudaSuccess &&
            cudaMalloc(&E->word, sizeof(unsigned long long) * nruns) == cudaSuccess &&
            cudaMalloc(&E->done, sizeof(unsigned int) * nruns) == cudaSuccess &&
            cudaMalloc(&E->remaining, sizeof(int) * 2) == cudaSuccess &&
            cudaMalloc(&E->lines, sizeof(EnsLine) * loff) == cudaSuccess &&
            cudaMalloc(&E->lines11, sizeof(EnsLine11) * loff) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    ens_free(E);
    return fail_msg(VLP4D_ERR_CUDA, "cudaMalloc failed in vlp4d_ensemble_create");
  }
  E->err = E->remaining + 1;
  if (cudaMemcpy(E->runs, E->host_runs.data(), sizeof(EnsRun) * nruns, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(E->F[1], 0, sizeof(float) * foff) != cudaSuccess ||
      cudaMemset(E->remaining, 0, sizeof(int) * 2) != cudaSuccess) {
    cudaGetLastError();
    ens_free(E);
    return fail_msg(VLP4D_ERR_CUDA, "ensemble upload failed");
  }
  k_ens_lines<<<nruns, 64>>>(E->runs, E->lines, E->lines11);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
    cudaGetLastError();
    ens_free(E);
    return fail_msg(VLP4D_ERR_CUDA, "ensemble line tables failed");
  }
  *out = E;
  return VLP4D_OK;
}

int vlp4d_ensemble_destroy(vlp4d_ensemble *ens) {
  if (!ens) return VLP4D_OK;
  cudaSetDevice(ens->device);
  cudaDeviceSynchronize();
  ens_free(ens);
  return VLP4D_OK;
}

int vlp4d_ensemble_set_tiles(vlp4d_ensemble *ens, int threads, int cols_per_tile, int ctas_per_sm) {
  if (!ens) return fail_msg(VLP4D_ERR_INVALID_ARG, "ens is NULL");
  if (threads < 32 || threads > 512 || threads % 32) return fail_msg(VLP4D_ERR_INVALID_ARG, "threads: a multiple of 32 in [32, 512]");
  if (cols_per_tile < 1 || cols_per_tile > threads) return fail_msg(VLP4D_ERR_INVALID_ARG, "cols_per_tile: in [1, threads]");
  if (ctas_per_sm < 0 || ctas_per_sm > 32) return fail_msg(VLP4D_ERR_INVALID_ARG, "ctas_per_sm: in [0, 32]");
  ens->threads = threads;
  ens->cc = cols_per_tile;
  ens->ctas_per_sm = ctas_per_sm;
  if (ens->graph) {
    cudaGraphExecDestroy(ens->graph);
    ens->graph = nullptr;
  }
  return VLP4D_OK;
}

int vlp4d_ensemble_set_idle_limit(vlp4d_ensemble *ens, long long cycles) {
  if (!ens) return fail_msg(VLP4D_ERR_INVALID_ARG, "ens is NULL");
  if (cycles < 0 || cycles > kEnsIdleLimit)
    return fail_msg(VLP4D_ERR_INVALID_ARG, "idle limit: 0 (default) or 1 .. 4e9 cycles");
  ens->idle_limit = cycles ? cycles : kEnsIdleLimit;
  if (ens->graph) {  // the graph holds the kernel's arguments: capture again
    cudaGraphExecDestroy(ens->graph);
    ens->graph = nullptr;
  }
  return VLP4D_OK;
}

int vlp4d_ensemble_get_tiles(const vlp4d_ensemble *ens, int *threads, int *cols_per_tile, int *ctas_per_sm) {
  if (!ens) return fail_msg(VLP4D_ERR_INVALID_ARG, "ens is NULL");
  if (threads) *threads = ens->threads;
  if (cols_per_tile) *cols_per_tile = ens->cc;
  if (ctas_per_sm) *ctas_per_sm = ens->ctas_per_sm;
  return VLP4D_OK;
}

int vlp4d_ensemble_run(vlp4d_ensemble *ens, void *stream) {
  if (!ens) return fail_msg(VLP4D_ERR_INVALID_ARG, "ens is NULL");
  EnsDeviceScope dev_scope(ens->device);
  if (!dev_scope.ok) return fail_msg(VLP4D_ERR_CUDA, "ensemble: cannot make its device current");
  vlp4d_ensemble *E = ens;
  cudaStream_t s = (cudaStream_t)stream;
  int rc;
  if (!E->graph) {
    // Capture on a private stream (the legacy stream cannot be captured).
    cudaStream_t cs;
    VLP4D_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
      cudaGetLastError();
      cudaStreamDestroy(cs);
      return fail_msg(VLP4D_ERR_CUDA, "ensemble: stream capture failed");
    }
    rc = ens_launch(E, E->nsteps, cs);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (rc || e != cudaSuccess || !g) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return rc ? rc : fail_msg(VLP4D_ERR_CUDA, "ensemble: stream capture failed");
    }
    const cudaError_t ie = cudaGraphInstantiate(&E->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      cudaGetLastError();
      E->graph = nullptr;
      return fail_msg(VLP4D_ERR_CUDA, std::string("ensemble: cudaGraphInstantiate: ") + cudaGetErrorString(ie));
    }
  }
  VLP4D_CUDA_TRY(cudaGraphLaunch(E->graph, s));
  return VLP4D_OK;
}

int vlp4d_ensemble_check(vlp4d_ensemble *ens) {
  if (!ens) return fail_msg(VLP4D_ERR_INVALID_ARG, "ens is NULL");
  EnsDeviceScope dev_scope(ens->device);
  if (!dev_scope.ok) return fail_msg(VLP4D_ERR_CUDA, "ensemble: cannot make its device current");
  VLP4D_CUDA_TRY(cudaDeviceSynchronize());
  return ens_check(ens);
}

int vlp4d_ensemble_read(vlp4d_ensemble *ens, int run, void *f_out, double *nrj, void *stream) {
  if (!ens) return fail_msg(VLP4D_ERR_INVALID_ARG, "ens is NULL");
  EnsDeviceScope dev_scope(ens->device);
  if (!dev_scope.ok) return fail_msg(VLP4D_ERR_CUDA, "ensemble: cannot make its device current");
  if (run < 0 || run >= ens->nruns) return fail_msg(VLP4D_ERR_INVALID_ARG, "run index out of range");
  const EnsRun &R = ens->host_runs[run];
  cudaStream_t s = (cudaStream_t)stream;
  const long long cells = (long long)R.n[0] * R.n[1] * R.n[2] * R.n[3];
  if (f_out)
    VLP4D_CUDA_TRY(cudaMemcpyAsync(f_out, ens->F[ens->nsteps > 0 ? 1 : 0] + R.f_off, sizeof(float) * cells,
                                   cudaMemcpyDeviceToDevice, s));
  if (nrj) {
    VLP4D_CUDA_TRY(cudaMemcpyAsync(nrj, ens->nrj + R.d_off, sizeof(double) * (ens->nsteps + 1),
                                   cudaMemcpyDeviceToHost, s));
    VLP4D_CUDA_TRY(cudaStreamSynchronize(s));
  }
  return VLP4D_OK;
}

long long vlp4d_ensemble_cells(const vlp4d_ensemble *ens) { return ens ? ens->total_cells : 0; }

// Scans thread counts {128, 256, 512}, columns per v tile {8, 16, 32, 64}
// and CTAs per SM {1, 2, 3, 4} (those that fit), timing `steps` steps of
// the ensemble for each (CUDA events, best of two), appends one CSV line per
// configuration to csv_path (when not NULL) and keeps the fastest.
int vlp4d_ensemble_autotune(vlp4d_ensemble *ens, int steps, const char *csv_path, void *stream) {
  if (!ens) return fail_msg(VLP4D_ERR_INVALID_ARG, "ens is NULL");
  EnsDeviceScope dev_scope(ens->device);
  if (!dev_scope.ok) return fail_msg(VLP4D_ERR_CUDA, "ensemble: cannot make its device current");
  if (steps < 1 || steps > ens->nsteps) steps = ens->nsteps > 0 ? ens->nsteps : 1;
  vlp4d_ensemble *E = ens;
  cudaStream_t s = (cudaStream_t)stream;
  FILE *csv = csv_path ? fopen(csv_path, "w") : nullptr;
  if (csv_path && !csv) return fail_msg(VLP4D_ERR_IO, std::string("cannot write ") + csv_path);
  if (csv) fprintf(csv, "threads,cols_per_tile,ctas_per_sm,steps,ms\n");
  cudaEvent_t e0, e1;
  VLP4D_CUDA_TRY(cudaEventCreate(&e0));
  VLP4D_CUDA_TRY(cudaEventCreate(&e1));
  const int th_list[3] = {128, 256, 512}, cc_list[4] = {8, 16, 32, 64}, cps_list[4] = {1, 2, 3, 4};
  float best = 1e30f;
  int bt = E->threads, bc = E->cc, bp = E->ctas_per_sm;
  int rc = VLP4D_OK;
  VLP4D_CUDA_TRY(cudaFuncSetAttribute(k_ensemble, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)E->smem));
  for (int th : th_list)
    for (int cc : cc_list) {
      if (cc > th) continue;
      for (int cps : cps_list) {
        int fit = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, k_ensemble, th, E->smem) != cudaSuccess) {
          cudaGetLastError();
          continue;
        }
        if (cps > fit) continue;
        E->threads = th;
        E->cc = cc;
        E->ctas_per_sm = cps;
        float ms = 1e30f;
        for (int rep = 0; rep < 2 && rc == VLP4D_OK; ++rep) {
          cudaEventRecord(e0, s);
          rc = ens_launch(E, steps, s);
          cudaEventRecord(e1, s);
          if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail_msg(VLP4D_ERR_CUDA, "ensemble autotune: launch failed");
          float t = 0.f;
          cudaEventElapsedTime(&t, e0, e1);
          if (t < ms) ms = t;
        }
        if (rc == VLP4D_OK) rc = ens_check(E);
        if (rc) break;
        if (csv) fprintf(csv, "%d,%d,%d,%d,%.4f\n", th, cc, cps, steps, ms);
        if (ms < best) {
          best = ms;
          bt = th;
          bc = cc;
          bp = cps;
        }
      }
      if (rc) break;
    }
  if (csv) fclose(csv);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  E->threads = bt;
  E->cc = bc;
  E->ctas_per_sm = bp;
  if (E->graph) {
    cudaGraphExecDestroy(E->graph);
    E->graph = nullptr;
  }
  return rc;
}

}  // extern "C"
