// Fused vx/vy advection pass over column chunks.
//
// Replaces advect_1D_vx followed by advect_1D_vy (miniapps/vlp4d/thrust/
// advection.hpp:203-328, run back to back in timestep.hpp:40-48).
//
// For a fixed spatial point (ix, iy) both velocity shifts are constant
// (dt*Ex(ix,iy) and dt*Ey(ix,iy)), so each "column" ixy = ix + nx*iy has one
// vx stencil and one vy stencil, read from the device-built line tables.  A
// work item is a chunk of C consecutive columns (C*elem = 128 bytes) and a
// segment of Q output vy rows.  The kernel streams "slabs" f[ixy0:ixy0+C,
// :, ivy] (C x nvx elements, one 3D TMA tile, layout [ivx][c]) through a
// `stages`-deep mbarrier pipeline, in vy order starting at the smallest
// vy offset of the chunk.  Each thread owns one column and V consecutive vx:
// it applies the vx stencil to every slab (taps from shared memory; the bank
// depends only on the column, so per-column offsets never conflict), keeps
// the last six vx-swept rows in registers and emits output row ivy once the
// six rows ivy+o..ivy+o+5 of its own column's vy offset o are in the window.
// Stores of a warp cover C consecutive columns: 128 contiguous bytes.  In
// FP32 a thread evaluates its vx rows i and i+V/2 as one packed pair (same
// column, same weights), with the f32x2 instructions.
#include <cudaTypedefs.h>

#include "internal.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace vlp4d {

namespace {

constexpr int kMaxStages = 12;
// Header ahead of the slabs: kMaxStages full barriers (8 B each), kMaxStages
// release counters and the issued-slab counter (4 B each).
constexpr int kBarBytes = 256;
static_assert(8 * kMaxStages + 4 * kMaxStages + 4 <= kBarBytes, "slab header overflow");

struct VslabArgs {
  void *fout;
  int nxy, nvx;
  int nvy;    // period of the vy offsets (the run's nvy; for slab contexts the global one)
  // Input rows: row0 < 0, periodic rows (start + t) mod nvy; row0 >= 0 (slab
  // contexts), rows start + t + row0 of an input of nin planes (the owned
  // planes and `row0` halo planes on each side), never wrapped.
  int row0, nin;
  int C;      // columns per chunk
  int Q;      // output vy rows per item (divides nvy)
  int nseg;   // nvy / Q
  long long nitems;
  int stages;
  StencilTable tvx, tvy;
  const int2 *span;  // per chunk: (min, max) signed vy offset of its columns
  int *err;
  // Per-column term added to every output of the column (kernels with
  // BIAS only): out += bias_scale * bias[ixy], the reverse mode's field term.
  const double *bias;
  double bias_scale;
};


// Error exit of one warp after a copy timed out: flag it, let the copies
// already issued for slabs k .. issued-1 land (bounded waits), then leave.
// The other warps reach their own time limits on the slabs this warp no
// longer releases and leave the same way.
__device__ __noinline__ void vslab_abort(const VslabArgs &a, uint64_t *bars, const int *issued, long long k, int S) {
  if ((threadIdx.x & 31) == 0) {
    atomicExch(a.err, 1);
    const long long n = *(volatile const int *)issued;
    for (long long q = k; q < n; ++q) mbar_wait_bounded(&bars[q % S], (uint32_t)((q / S) & 1));
  }
  __syncwarp();
}

// FP64 vx sweep of V outputs from V+5 taps (the FP32 path is packed inline).
template <int V>
__device__ __forceinline__ void vx_sweep(const double (&t)[V + 5], const double (&w)[6], double (&o)[V]) {
#pragma unroll
  for (int i = 0; i < V; ++i) o[i] = interp6(w, t[i], t[i + 1], t[i + 2], t[i + 3], t[i + 4], t[i + 5]);
}

// Position in the CTA's slab sequence: item, slab index within the item,
// slab count and first vy row of the item, column chunk.  Every warp keeps
// an identical cursor S slabs ahead of the slab it consumes, so whichever
// warp releases a slot last can refill it without asking anyone.
struct SlabCursor {
  long long item;
  int t, cnt, start, cc;
};

template <bool DVY>
__device__ __forceinline__ void cursor_item(const VslabArgs &a, SlabCursor &c) {
  if (c.item >= a.nitems) return;
  c.cc = (int)(c.item / a.nseg);
  const int sg = (int)(c.item % a.nseg);
  if (DVY) {
    const int2 sp = a.span[c.cc];
    c.cnt = a.Q + (sp.y - sp.x) + 5;
    c.start = sg * a.Q + sp.x;
  } else {
    c.cnt = a.Q;
    c.start = sg * a.Q;
  }
}

template <bool DVY>
__device__ __forceinline__ void cursor_next(const VslabArgs &a, SlabCursor &c) {
  if (c.item >= a.nitems) return;
  if (++c.t == c.cnt) {
    c.t = 0;
    c.item += gridDim.x;
    cursor_item<DVY>(a, c);
  }
}

// SLAB: the input rows of a slab context (owned planes and halos, never
// wrapped); otherwise periodic rows.  A separate instantiation, so that the
// periodic kernels carry none of the slab arithmetic.
template <typename T, bool SLAB = false>
__device__ __forceinline__ void issue_slab(const CUtensorMap *tin, const VslabArgs &a, const SlabCursor &c,
                                           T *slabs, uint64_t *bars, int slot, size_t slab_elems,
                                           uint32_t slab_bytes) {
  int row = c.start + c.t;
  if constexpr (!SLAB) {
    row %= a.nvy;
    if (row < 0) row += a.nvy;
  } else {
    row += a.row0;
    if (row < 0 || row >= a.nin) {  // the halo is too narrow for this column's shift
      atomicOr(a.err, kErrSlabHalo);
      row = row < 0 ? 0 : a.nin - 1;
    }
  }
  mbar_arrive_expect_tx(&bars[slot], slab_bytes);
  tensor_load_3d(slabs + (size_t)slot * slab_elems, tin, c.cc * a.C, 0, row, &bars[slot]);
}

// NXY: compile-time nx*ny (0 = read a.nxy at run time); with it the V output
// stores of a thread use immediate offsets.
template <typename T, bool DVX, bool DVY, int V, int NXY, bool BIAS = false, bool SLAB = false>
__global__ void __launch_bounds__(512) k_vslab(const __grid_constant__ CUtensorMap tin, VslabArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // Tensor-copy destinations on a 128-byte boundary whatever the base
  // alignment of dynamic shared memory (the launch adds 128 bytes of slack).
  unsigned char *smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  const int C = a.C, nvx = a.nvx, S = a.stages;
  const size_t slab_elems = (size_t)C * nvx;
  const uint32_t slab_bytes = (uint32_t)(slab_elems * sizeof(T));
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);          // S full barriers
  int *released = reinterpret_cast<int *>(smem + 8 * kMaxStages);  // S release counters
  int *issued = released + kMaxStages;                          // slabs issued so far
  T *slabs = reinterpret_cast<T *>(smem + kBarBytes);
  const int col = threadIdx.x % C;
  const int vx0 = (threadIdx.x / C) * V;
  const int lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&bars[s], 1);
      released[s] = 0;
    }
    mbar_fence_init();
  }
  __syncthreads();

  // Look-ahead cursor: slab S of the sequence (the first S are issued here).
  SlabCursor ahead;
  ahead.item = blockIdx.x;
  ahead.t = 0;
  cursor_item<DVY>(a, ahead);
  if (threadIdx.x == 0) {
    int n = 0;
    for (; n < S && ahead.item < a.nitems; ++n) {
      issue_slab<T, SLAB>(&tin, a, ahead, slabs, bars, n, slab_elems, slab_bytes);
      cursor_next<DVY>(a, ahead);
    }
    *issued = n;
  } else {
    for (int n = 0; n < S && ahead.item < a.nitems; ++n) cursor_next<DVY>(a, ahead);
  }

  const long long vstride = NXY ? NXY : a.nxy;            // consecutive ivx
  const long long ystride = vstride * nvx;                 // consecutive ivy
  long long k = 0;                                         // slabs consumed
  int slot = 0;                                            // k % S
  uint32_t parity = 0;                                     // (k / S) & 1
  for (long long item = blockIdx.x; item < a.nitems; item += gridDim.x) {
    SlabCursor cur;
    cur.item = item;
    cur.t = 0;
    cursor_item<DVY>(a, cur);
    const int cnt = cur.cnt, cc = cur.cc;
    const int sg = (int)(item % a.nseg);
    const long long ixy = (long long)cc * C + col;
    T wvx[6], wvy[6];
    int lag0 = 0;
    // Shared-memory offsets of this thread's V+5 vx taps ([ivx][c] layout),
    // the same for every slab of the item.
    int off[V + 5];
    {
      int j = vx0;
      if (DVX) {
        j += __ldg(a.tvx.m + ixy);
        if (j >= nvx) j -= nvx;
        load_weights(WeightsOf<T>::get(a.tvx), ixy, wvx);
      }
#pragma unroll
      for (int q = 0; q < V + 5; ++q) {
        off[q] = j * C + col;
        if (++j == nvx) j = 0;
      }
    }
    if (DVY) {
      lag0 = 5 + signed_offset(__ldg(a.tvy.m + ixy), a.nvy) - a.span[cc].x;
      load_weights(WeightsOf<T>::get(a.tvy), ixy, wvy);
    }
    constexpr bool has_bias = BIAS;
    const double bias = BIAS ? a.bias_scale * __ldg(a.bias + ixy) : 0.0;
    // Output pointer of the next row this thread writes.
    T *orow = static_cast<T *>(a.fout) + ixy + vstride * vx0 + ystride * (long long)sg * a.Q;
    // Ring of vx-swept rows, slot = t % 6 (static after unrolling).  FP64:
    // win[slot][i] is vx row vx0+i.  FP32: packed pairs, win2[slot][i] holds
    // vx rows (vx0+i, vx0+i+V/2), which share the column's weights.
    constexpr int H = V / 2;
    constexpr bool kF32 = sizeof(T) == 4;
    T win[6][kF32 ? 1 : V];
    float2 win2[6][kF32 ? H : 1];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
#pragma unroll
      for (int i = 0; i < (kF32 ? 1 : V); ++i) win[j][i] = T(0);
#pragma unroll
      for (int i = 0; i < (kF32 ? H : 1); ++i) win2[j][i] = make_float2(0.f, 0.f);
    }
    SweepW<float> svx, svy;
    if constexpr (kF32) {
      if (DVX) make_sweep_w(reinterpret_cast<const float(&)[6]>(wvx), svx);
      if (DVY) make_sweep_w(reinterpret_cast<const float(&)[6]>(wvy), svy);
    }

    for (int t0 = 0; t0 < cnt; t0 += 6) {
#pragma unroll
      for (int u = 0; u < 6; ++u) {
        const int t = t0 + u;
        if (t >= cnt) break;  // uniform over the CTA
        if (!mbar_wait_bounded(&bars[slot], parity)) {
          vslab_abort(a, bars, issued, k, S);
          return;
        }
        const T *sl = slabs + (size_t)slot * slab_elems;
        if constexpr (kF32) {
          const float *slf = reinterpret_cast<const float *>(sl);
          if (DVX) {
            // P[k] = (tap k, tap k+H); D[k] = (d_k, d_{k+H}), d_k = tap k+1 - tap k.
            float2 P[H + 5], D[H + 4];
#pragma unroll
            for (int q = 0; q < H + 5; ++q) P[q] = make_float2(slf[off[q]], slf[off[q + H]]);
#pragma unroll
            for (int q = 0; q < H + 4; ++q) D[q] = sub2(P[q + 1], P[q]);
#pragma unroll
            for (int i = 0; i < H; ++i) win2[u][i] = interp_diff2(svx.v, P[i + 2], D[i], D[i + 1], D[i + 2], D[i + 3], D[i + 4]);
          } else {
#pragma unroll
            for (int i = 0; i < H; ++i) win2[u][i] = make_float2(slf[off[i]], slf[off[i + H]]);
          }
        } else {
          if (DVX) {
            T tap[V + 5];
#pragma unroll
            for (int q = 0; q < V + 5; ++q) tap[q] = sl[off[q]];
            vx_sweep<V>(tap, wvx, win[u]);
          } else {
#pragma unroll
            for (int i = 0; i < V; ++i) win[u][i] = sl[off[i]];
          }
        }
        // This warp is done with the slot: count it; the last warp refills it.
        __syncwarp();
        if (lane == 0) {
          __threadfence_block();
          if (atomicAdd(&released[slot], 1) == nwarps - 1) {
            released[slot] = 0;
            __threadfence_block();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            if (ahead.item < a.nitems) {
              issue_slab<T, SLAB>(&tin, a, ahead, slabs, bars, slot, slab_elems, slab_bytes);
              atomicAdd(issued, 1);
            }
          }
        }
        cursor_next<DVY>(a, ahead);
        bool emit = true;
        if (DVY) {
          const int e = t - lag0;
          emit = e >= 0 && e < a.Q;
        }
        if (emit) {
          if constexpr (kF32) {
            float *orowf = reinterpret_cast<float *>(orow);
#pragma unroll
            for (int i = 0; i < H; ++i) {
              float2 val;
              if (DVY) {  // rows t-5 .. t sit in slots u+1 .. u+6 (mod 6)
                const float2 f0 = win2[(u + 1) % 6][i], f1 = win2[(u + 2) % 6][i], f2 = win2[(u + 3) % 6][i],
                             f3 = win2[(u + 4) % 6][i], f4 = win2[(u + 5) % 6][i], f5 = win2[u][i];
                val = interp_diff2(svy.v, f2, sub2(f1, f0), sub2(f2, f1), sub2(f3, f2), sub2(f4, f3), sub2(f5, f4));
              } else {
                val = win2[u][i];
              }
              if constexpr (has_bias) {
                val.x = (float)((double)val.x + bias);
                val.y = (float)((double)val.y + bias);
              }
              orowf[vstride * i] = val.x;
              orowf[vstride * (i + H)] = val.y;
            }
          } else {
#pragma unroll
            for (int i = 0; i < V; ++i) {
              T val;
              if (DVY)  // rows t-5 .. t sit in slots u+1 .. u+6 (mod 6)
                val = interp6(wvy, win[(u + 1) % 6][i], win[(u + 2) % 6][i], win[(u + 3) % 6][i],
                              win[(u + 4) % 6][i], win[(u + 5) % 6][i], win[u][i]);
              else
                val = win[u][i];
              if constexpr (has_bias) val = (T)((double)val + bias);
              orow[vstride * i] = val;
            }
          }
          orow += ystride;
        }
        ++k;
        if (++slot == S) {
          slot = 0;
          parity ^= 1u;
        }
      }
    }
  }
}

// Per column chunk of C columns: smallest and largest signed vy offset.
__global__ void k_vspan(const int *__restrict__ mvy, int nchunks, int C, int nvy, int2 *__restrict__ span) {
  const int cc = blockIdx.x * blockDim.x + threadIdx.x;
  if (cc >= nchunks) return;
  int lo = 1 << 30, hi = -(1 << 30);
  for (int c = 0; c < C; ++c) {
    const int o = signed_offset(mvy[(long long)cc * C + c], nvy);
    lo = o < lo ? o : lo;
    hi = o > hi ? o : hi;
  }
  span[cc] = make_int2(lo, hi);
}

}  // namespace
}  // namespace vlp4d

namespace vlp4d {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  }
  return fn;
}

int env_int(const char *name, int dflt) {
  const char *v = getenv(name);
  return v && *v ? atoi(v) : dflt;
}

struct VslabCfg {
  int C = 0, V = 0, Q = 0, stages = 0, threads = 0;
  size_t smem = 0;
};

// C*elem = 128 bytes per slab row (64 when nvx > 128), V vx per thread,
// 512 threads.  Q output rows per item (the segment height, below): each
// item re-reads the 5 + spread halo slabs of its vy segment (4% at Q = 128,
// 8% at 64; at 128^4: 64 in FP32, 128 in FP64, whose chunks are half as
// wide).  Stages as measured best at
// 128^4: 8 for the FP32 vx+vy pass (one 512-thread CTA per SM, by
// registers), 4 for a single FP32 direction (lighter threads: four stages
// leave room for several CTAs per SM; 0.46 -> 0.38 ms for vx, 0.50 -> 0.41
// ms for vy), 4 in FP64.  VLP4D_VSLAB_Q and VLP4D_VSLAB_STAGES override for
// tuning sweeps.
bool vslab_config(const vlp4d_ctx *c, bool do_vx, bool do_vy, VslabCfg &cfg) {
  const bool both = do_vx && do_vy;
  const long long nxy = c->g.nxy();
  const int nvx = c->g.n[2], nvy = c->g.n[3];
  const bool f32 = c->dtype == VLP4D_F32;
  if (nvx < 8 || nvx > 256) return false;
  cfg.V = f32 ? 8 : 4;
  cfg.C = vslab_chunk_cols(c);
  if (!cfg.C || nvx % cfg.V || nxy % cfg.C) return false;
  cfg.threads = cfg.C * (nvx / cfg.V);
  // Whole warps only: every warp releases each slab once, and the last of
  // blockDim/32 releases refills it.
  if (cfg.threads > 512 || cfg.threads < 32 || cfg.threads % 32) return false;
  // Q: the vy segment height.  A CTA streams its items one after another,
  // each item Q output rows plus (with a vy sweep) the five halo rows and
  // the chunk's offset spread, about Q + 6 slabs, and about four slab times
  // of start-up (tables, the pipeline refilling); with one CTA per SM the
  // pass takes about ceil(items / SMs) * (Q + halo + 4) slab times.  Q
  // minimises that among the divisors of nvy up to 128 that still give
  // every SM an item (the smallest Q when none does).  128^4 FP32: Q = 64
  // (1024 items, 7 per SM); 64^4 FP32: Q = 32 (60.8 -> 47.6 us for vx+vy
  // against Q = 8).
  const long long nchunks = nxy / cfg.C;
  int Q = env_int("VLP4D_VSLAB_Q", 0);
  if (Q <= 0) {
    Q = 0;
    long long best = -1;
    const int halo = do_vy ? 6 : 0;
    for (int q = nvy < 128 ? nvy : 128; q >= 1; --q) {
      if (nvy % q) continue;
      const long long items = nchunks * (nvy / q);
      if (items < c->num_sms && q != 1) continue;
      const long long cost = (items + c->num_sms - 1) / c->num_sms * (q + halo + 4);
      if (best < 0 || cost < best) {
        best = cost;
        Q = q;
      }
    }
    if (!Q) Q = 1;
  }
  if (Q > nvy) Q = nvy;
  while (Q > 1 && nvy % Q) --Q;
  cfg.Q = Q;
  cfg.stages = env_int("VLP4D_VSLAB_STAGES", f32 && both ? 8 : 4);
  if (cfg.stages < 2 || cfg.stages > kMaxStages) return false;
  cfg.smem = 128 + kBarBytes + (size_t)cfg.stages * cfg.C * nvx * c->elem;
  return cfg.smem <= 200 * 1024;
}

template <typename T, bool DVX, bool DVY, int V, int NXY, bool BIAS = false, bool SLAB = false>
int run_vslab(vlp4d_ctx *c, const CUtensorMap &map, const VslabArgs &args, const VslabCfg &cfg, cudaStream_t s) {
  auto kern = k_vslab<T, DVX, DVY, V, NXY, BIAS, SLAB>;
  VLP4D_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem));
  int per_sm = 0;
  VLP4D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, cfg.threads, cfg.smem));
  if (per_sm < 1) return VLP4D_ERR_UNSUPPORTED;
  // At most 512 threads per SM (VLP4D_VSLAB_CTAS sets the CTAs per SM):
  // where registers allow more (the FP64 vx sweep alone, 64 registers, two
  // CTAs of 512 threads) the pass measured slower, 0.86 against 0.74 ms at
  // 128^4; blocks of 256 threads (64^4) keep two CTAs per SM.
  const int cap = env_int("VLP4D_VSLAB_CTAS", 512 / cfg.threads > 0 ? 512 / cfg.threads : 1);
  if (cap > 0 && per_sm > cap) per_sm = cap;
  long long grid = (long long)per_sm * c->num_sms;
  if (grid > args.nitems) grid = args.nitems;
  kern<<<(unsigned)grid, cfg.threads, cfg.smem, s>>>(map, args);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

}  // namespace

int launch_advect_vxvy(vlp4d_ctx *c, const void *fn, void *fnp1, bool do_vx, bool do_vy, cudaStream_t s) {
  return launch_advect_vxvy_tables(c, fn, fnp1, do_vx ? &c->tab_vx : nullptr, do_vy ? &c->tab_vy : nullptr, s);
}

int vslab_chunk_cols(const vlp4d_ctx *c) {
  const int nvx = c->g.n[2];
  if (nvx < 8 || nvx > 256) return 0;
  const int C = c->dtype == VLP4D_F32 ? (nvx <= 128 ? 32 : 16) : (nvx <= 128 ? 16 : 8);
  return c->g.nxy() % C ? 0 : C;
}

int launch_advect_vxvy_tables(vlp4d_ctx *c, const void *fn, void *fnp1, const StencilTable *tvx,
                              const StencilTable *tvy, cudaStream_t s, const double *bias, double bias_scale) {
  const bool do_vx = tvx != nullptr, do_vy = tvy != nullptr;
  if (!c->fused) return VLP4D_ERR_UNSUPPORTED;
  if (((uintptr_t)fn & 15) || ((uintptr_t)fnp1 & 15)) return VLP4D_ERR_UNSUPPORTED;
  if (!do_vx && !do_vy) return VLP4D_ERR_UNSUPPORTED;
  VslabCfg cfg;
  if (!vslab_config(c, do_vx, do_vy, cfg)) return VLP4D_ERR_UNSUPPORTED;
  PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode) return VLP4D_ERR_UNSUPPORTED;
  const long long nxy = c->g.nxy();
  const int nvx = c->g.n[2], nvy = c->g.n[3];
  const size_t elem = c->elem;
  const int nchunks = (int)(nxy / cfg.C);
  if (do_vy && nchunks > c->vspan_cap) return VLP4D_ERR_UNSUPPORTED;
  // Slab contexts with a vy sweep read the whole input buffer (owned planes
  // and both halos) and write the owned planes; everything else reads and
  // writes nvy planes.
  const bool slab_in = c->slab && do_vy;
  const int nin = slab_in ? nvy + 2 * c->halo : nvy;

  CUtensorMap map;
  cuuint64_t dims[3] = {(cuuint64_t)nxy, (cuuint64_t)nvx, (cuuint64_t)nin};
  cuuint64_t strides[2] = {(cuuint64_t)(nxy * elem), (cuuint64_t)(nxy * nvx * elem)};
  cuuint32_t box[3] = {(cuuint32_t)cfg.C, (cuuint32_t)nvx, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode(&map, elem == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                      const_cast<void *>(fn), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return VLP4D_ERR_UNSUPPORTED;

  // The chunks' vy spans: from the table when its builder made them for
  // this chunk width, else here.
  const int2 *span = c->vspan;
  if (do_vy && tvy->span && tvy->span_C == cfg.C) {
    span = tvy->span;
  } else if (do_vy) {
    k_vspan<<<(nchunks + 127) / 128, 128, 0, s>>>(tvy->m, nchunks, cfg.C, c->nvy_glob, c->vspan);
    VLP4D_LAUNCH_CHECK();
  }
  VslabArgs a;
  a.fout = fnp1;
  a.nxy = (int)nxy;
  a.nvx = nvx;
  a.nvy = slab_in ? c->nvy_glob : nvy;
  a.row0 = slab_in ? c->halo : -1;
  a.nin = nin;
  a.C = cfg.C;
  a.Q = cfg.Q;
  a.nseg = nvy / cfg.Q;
  a.nitems = (long long)nchunks * a.nseg;
  a.stages = cfg.stages;
  if (do_vx) a.tvx = *tvx;
  if (do_vy) a.tvy = *tvy;
  a.span = span;
  a.err = c->d_err;
  a.bias = bias;
  a.bias_scale = bias_scale;
#define VLP4D_VS(T, DVX, DVY, V)                                                  \
  switch (a.nxy) {                                                                \
    case 16384: return run_vslab<T, DVX, DVY, V, 16384>(c, map, a, cfg, s);      \
    case 4096: return run_vslab<T, DVX, DVY, V, 4096>(c, map, a, cfg, s);        \
    default: return run_vslab<T, DVX, DVY, V, 0>(c, map, a, cfg, s);             \
  }
  if (slab_in) {  // slab contexts: rows of the owned planes and halos
    if (bias) return VLP4D_ERR_UNSUPPORTED;
    if (c->dtype == VLP4D_F64) {
      if (do_vx) return run_vslab<double, true, true, 4, 0, false, true>(c, map, a, cfg, s);
      return run_vslab<double, false, true, 4, 0, false, true>(c, map, a, cfg, s);
    }
    if (do_vx) return run_vslab<float, true, true, 8, 0, false, true>(c, map, a, cfg, s);
    return run_vslab<float, false, true, 8, 0, false, true>(c, map, a, cfg, s);
  }
  if (bias) {  // the reverse mode's vx+vy pass with the per-column term
    if (!(do_vx && do_vy)) return VLP4D_ERR_UNSUPPORTED;
    if (c->dtype == VLP4D_F64) return run_vslab<double, true, true, 4, 0, true>(c, map, a, cfg, s);
    switch (a.nxy) {  // the plane sizes of the benchmark configurations, compile-time
      case 16384: return run_vslab<float, true, true, 8, 16384, true>(c, map, a, cfg, s);
      case 4096: return run_vslab<float, true, true, 8, 4096, true>(c, map, a, cfg, s);
      default: return run_vslab<float, true, true, 8, 0, true>(c, map, a, cfg, s);
    }
  }
  if (c->dtype == VLP4D_F64) {
    if (do_vx && do_vy) VLP4D_VS(double, true, true, 4);
    if (do_vx) VLP4D_VS(double, true, false, 4);
    VLP4D_VS(double, false, true, 4);
  } else {
    if (do_vx && do_vy) VLP4D_VS(float, true, true, 8);
    if (do_vx) VLP4D_VS(float, true, false, 8);
    VLP4D_VS(float, false, true, 8);
  }
#undef VLP4D_VS
}

}  // namespace vlp4d
