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
  int rt;      // output rows per thread task in phase Y (divides R)
  StencilTable tx, ty;
  double *rho_part;  // [G][nx*ny] partial moments, when the moment is fused
  int *err;
};

// Elements a0..a0+11 (mod nx) of a shared row, a0 a multiple of 4, nx a
// multiple of 4: three aligned 4-vectors, so no access straddles the wrap.
template <typename T>
__device__ __forceinline__ void load12(const T *row, int a0, int nx, T (&v)[12]) {
  T q[4];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    load4(row + a0, q);
#pragma unroll
    for (int i = 0; i < 4; ++i) v[4 * b + i] = q[i];
    a0 += 4;
    if (a0 >= nx) a0 -= nx;
  }
}

// Four x-swept outputs at columns c0..c0+3 of one staged row; r = (c0+mx)%4
// is uniform over the CTA, so the switch does not diverge.
template <typename T>
__device__ __forceinline__ void sweep_x4(const T *row, int c0, int mx, int nx, const T (&w)[6], T (&o)[4]) {
  int base = c0 + mx;
  if (base >= nx) base -= nx;
  const int r = base & 3;
  T v[12];
  load12(row, base - r, nx, v);
#define VLP4D_SX(R_)                                                                                 \
  _Pragma("unroll") for (int q = 0; q < 4; ++q) o[q] =                                              \
      interp6(w, v[R_ + q], v[R_ + q + 1], v[R_ + q + 2], v[R_ + q + 3], v[R_ + q + 4], v[R_ + q + 5])
  switch (r) {
    case 0: VLP4D_SX(0); break;
    case 1: VLP4D_SX(1); break;
    case 2: VLP4D_SX(2); break;
    default: VLP4D_SX(3); break;
  }
#undef VLP4D_SX
}

__device__ __forceinline__ void rho_add4(double *p, const float (&o)[4]) {
  double2 a = reinterpret_cast<double2 *>(p)[0], b = reinterpret_cast<double2 *>(p)[1];
  a.x += (double)o[0]; a.y += (double)o[1]; b.x += (double)o[2]; b.y += (double)o[3];
  reinterpret_cast<double2 *>(p)[0] = a;
  reinterpret_cast<double2 *>(p)[1] = b;
}
__device__ __forceinline__ void rho_add4(double *p, const double (&o)[4]) {
  double2 a = reinterpret_cast<double2 *>(p)[0], b = reinterpret_cast<double2 *>(p)[1];
  a.x += o[0]; a.y += o[1]; b.x += o[2]; b.y += o[3];
  reinterpret_cast<double2 *>(p)[0] = a;
  reinterpret_cast<double2 *>(p)[1] = b;
}

template <typename T, bool DX, bool DY, bool RHO>
__global__ void __launch_bounds__(512) k_plane(PlaneArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int nx = a.nx, ny = a.ny, R = a.R, S = a.stages;
  const int vrows = R + a.halo;
  const size_t slot_elems = (size_t)vrows * nx;
  const uint32_t slot_bytes = (uint32_t)(slot_elems * sizeof(T));
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  T *slots = reinterpret_cast<T *>(smem + kBarBytes);
  T *xs = slots + (size_t)S * slot_elems;  // x-swept rows (x and y both on)
  double *rho_s = reinterpret_cast<double *>(xs + ((DX && DY) ? slot_elems : 0));

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
  if (RHO)
    for (int e = threadIdx.x; e < R * nx; e += blockDim.x) rho_s[e] = 0.0;
  __syncthreads();

  // Thread 0: stage the R + halo input rows of item `it` into its slot.
  auto issue = [&](long long it) {
    const long long p = g + it * G;
    int phys = chunk * R;
    if (DY) {
      phys += a.ty.m[(int)(p / a.nvx)];
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

  const int ncg = nx >> 2;
  for (long long it = 0; it < n_items; ++it) {
    const int slot = (int)(it % S);
    const bool ok = mbar_wait_bounded(&bars[slot], (uint32_t)((it / S) & 1));
    const long long p = g + it * G;
    const int ivx = (int)(p % a.nvx), ivy = (int)(p / a.nvx);
    const T *in = slots + (size_t)slot * slot_elems;
    T *outp = static_cast<T *>(a.fout) + p * plane_elems + (long long)chunk * R * nx;
    T wx[6], wy[6];
    int mx = 0;
    if (DX) {
      mx = __ldg(a.tx.m + ivx);
      load_weights(WeightsOf<T>::get(a.tx), ivx, wx);
    }
    if (DY) load_weights(WeightsOf<T>::get(a.ty), ivy, wy);

    if (DX) {  // Phase X: every staged row, four columns per task.
      const int tasks = vrows * ncg;
      for (int t = threadIdx.x; t < tasks; t += blockDim.x) {
        const int v = t / ncg, c0 = (t - v * ncg) * 4;
        T o[4];
        sweep_x4(in + (size_t)v * nx, c0, mx, nx, wx, o);
        if (DY) {
          store4(xs + (size_t)v * nx + c0, o);
        } else {
          store4(outp + (size_t)v * nx + c0, o);
          if (RHO) rho_add4(rho_s + (size_t)v * nx + c0, o);
        }
      }
    }
    if (DY) {  // Phase Y: rt consecutive output rows x four columns per task.
      if (DX) __syncthreads();
      const T *src = DX ? xs : in;
      const int rt = a.rt;
      const int tasks = (R / rt) * ncg;
      for (int t = threadIdx.x; t < tasks; t += blockDim.x) {
        const int rg = t / ncg, c0 = (t - rg * ncg) * 4, r0 = rg * rt;
        T w0[4], w1[4], w2[4], w3[4], w4[4], w5[4];
        load4(src + (size_t)(r0 + 0) * nx + c0, w1);
        load4(src + (size_t)(r0 + 1) * nx + c0, w2);
        load4(src + (size_t)(r0 + 2) * nx + c0, w3);
        load4(src + (size_t)(r0 + 3) * nx + c0, w4);
        load4(src + (size_t)(r0 + 4) * nx + c0, w5);
        for (int i = 0; i < rt; ++i) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            w0[q] = w1[q]; w1[q] = w2[q]; w2[q] = w3[q]; w3[q] = w4[q]; w4[q] = w5[q];
          }
          load4(src + (size_t)(r0 + i + 5) * nx + c0, w5);
          T o[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) o[q] = interp6(wy, w0[q], w1[q], w2[q], w3[q], w4[q], w5[q]);
          store4(outp + (size_t)(r0 + i) * nx + c0, o);
          if (RHO) rho_add4(rho_s + (size_t)(r0 + i) * nx + c0, o);
        }
      }
    }
    // Slot (and the x-swept buffer) are free once every thread is here.
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicExch(a.err, 1);
        const long long last = n_items < it + S ? n_items : it + S;
        for (long long k = it; k < last; ++k) mbar_wait_bounded(&bars[k % S], (uint32_t)((k / S) & 1));
      }
      __syncthreads();
      return;
    }
    if (threadIdx.x == 0 && it + S < n_items) issue(it + S);
  }
  if (RHO) {
    double *dst = a.rho_part + (long long)g * plane_elems + (long long)chunk * R * nx;
    for (int e = threadIdx.x; e < R * nx; e += blockDim.x) dst[e] = rho_s[e];
  }
}

}  // namespace
}  // namespace vlp4d

namespace vlp4d {

namespace {

struct PlaneCfg {
  int R = 0, rt = 1, stages = 3, threads = 0, cpp = 1, grid = 0, G = 0;
  size_t smem = 0;
};

int env_int(const char *name, int dflt) {
  const char *v = getenv(name);
  return v && *v ? atoi(v) : dflt;
}

size_t plane_smem(int R, int halo, int nx, size_t elem, int stages, bool dx, bool dy, bool rho) {
  const size_t slot = (size_t)(R + halo) * nx * elem;
  return kBarBytes + stages * slot + ((dx && dy) ? slot : 0) + (rho ? (size_t)R * nx * sizeof(double) : 0);
}

// Chooses the chunk height R (a divisor of ny), the pipeline depth and the
// block size.  Preference: the tallest chunk (least halo re-read) that still
// lets two CTAs share an SM, else one CTA per SM.  VLP4D_PLANE_R and
// VLP4D_PLANE_STAGES override the choice for tuning sweeps.
bool plane_config(const vlp4d_ctx *c, bool dx, bool dy, bool rho, PlaneCfg &cfg) {
  const int nx = c->g.n[0], ny = c->g.n[1];
  const size_t elem = c->elem;
  if (nx % 4 != 0 || nx > 2048) return false;
  const int halo = dy ? 5 : 0;
  cfg.stages = env_int("VLP4D_PLANE_STAGES", 3);
  if (cfg.stages < 2 || cfg.stages > kMaxStages) return false;
  const int forced = env_int("VLP4D_PLANE_R", 0);
  const size_t two_per_sm = 110 * 1024, one_per_sm = 220 * 1024;
  int best = 0;
  for (const size_t budget : {two_per_sm, one_per_sm}) {
    for (int R = ny < 64 ? ny : 64; R >= 1 && !best; --R) {
      if (ny % R) continue;
      if (forced && R != forced) continue;
      if (plane_smem(R, halo, nx, elem, cfg.stages, dx, dy, rho) <= budget) best = R;
    }
    if (best) break;
  }
  if (!best) return false;
  cfg.R = best;
  cfg.rt = best % 4 == 0 ? 4 : (best % 2 == 0 ? 2 : 1);
  cfg.cpp = ny / best;
  const int ytasks = dy ? (best / cfg.rt) * (nx / 4) : 0;
  const int xtasks = dx ? (best + halo) * (nx / 4) : 0;
  int threads = ytasks > 0 ? ytasks : xtasks;
  threads = ((threads + 31) / 32) * 32;
  if (threads < 64) threads = 64;
  if (threads > 512) threads = 512;
  cfg.threads = threads;
  cfg.smem = plane_smem(best, halo, nx, elem, cfg.stages, dx, dy, rho);
  return true;
}

template <typename T, bool DX, bool DY, bool RHO>
int run_plane(vlp4d_ctx *c, const PlaneArgs &args, PlaneCfg &cfg, cudaStream_t s) {
  auto kern = k_plane<T, DX, DY, RHO>;
  VLP4D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem));
  int per_sm = 0;
  VLP4D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, cfg.threads, cfg.smem));
  if (per_sm < 1) return VLP4D_ERR_UNSUPPORTED;
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
  if (!plane_config(c, do_x, do_y, with_rho, cfg)) return VLP4D_ERR_UNSUPPORTED;
  PlaneArgs a;
  a.fin = fn;
  a.fout = fnp1;
  a.nx = c->g.n[0];
  a.ny = c->g.n[1];
  a.nvx = c->g.n[2];
  a.nvy = c->g.n[3];
  a.R = cfg.R;
  a.cpp = cfg.cpp;
  a.halo = do_y ? 5 : 0;
  a.stages = cfg.stages;
  a.rt = cfg.rt;
  if (tx) a.tx = *tx;
  if (ty) a.ty = *ty;
  a.rho_part = c->rho_part;
  a.err = c->d_err;
  int rc;
#define VLP4D_PLANE(T, DX, DY, RHO) rc = run_plane<T, DX, DY, RHO>(c, a, cfg, s)
  if (c->dtype == VLP4D_F64) {
    if (do_x && do_y) { if (with_rho) VLP4D_PLANE(double, true, true, true); else VLP4D_PLANE(double, true, true, false); }
    else if (do_x) VLP4D_PLANE(double, true, false, false);
    else VLP4D_PLANE(double, false, true, false);
  } else {
    if (do_x && do_y) { if (with_rho) VLP4D_PLANE(float, true, true, true); else VLP4D_PLANE(float, true, true, false); }
    else if (do_x) VLP4D_PLANE(float, true, false, false);
    else VLP4D_PLANE(float, false, true, false);
  }
#undef VLP4D_PLANE
  if (rc) return rc;
  if (with_rho && do_x && do_y) return launch_rho_finish(c, cfg.G, s);
  if (with_rho) return launch_field_rho(c, fnp1, s);
  return VLP4D_OK;
}

}  // namespace vlp4d
