// Advection kernels of the vlp4d step: stencil tables and the generic
// (any-shape) sweeps.  The bandwidth-optimised plane and v-slab kernels live
// in advect_plane.cu and advect_vslab.cu and fall back to these when a shape
// is outside what they support.
//
// Reference: miniapps/vlp4d/thrust/advection.hpp:77-386 (four functors run
// by kernel_for_each_left over (ix, iy, ivx) with a serial ivy loop,
// lib/thrust/Cuda_Parallel_For.hpp:37-45).
#include <vector>

#include "internal.cuh"
#include "stencil.cuh"

namespace vlp4d {

namespace {

// One v-line per (ix, iy): displacement dt*E(ix, iy) (advection.hpp:243, 306).
// blockIdx.y selects the table (vx from Ex, vy from Ey), so that both are
// built by one launch.
struct VtableJob {
  const double *e;
  double hmin, hmax;
  int n;
  int *m;
  double *w;
  float *wf;
  int2 *span;  // non-null: also the chunk spans of the signed offsets (chunks of C lines)
  int C;
};
__global__ void k_build_vtable(VtableJob j0, VtableJob j1, int lines, double dt) {
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  const bool on = line < lines;
  const VtableJob j = blockIdx.y ? j1 : j0;
  int m = 0;
  if (on) {
    const LineStencil s = line_stencil(__dmul_rn(dt, j.e[line]), j.hmin, j.hmax, j.n);
    m = s.m;
    j.m[line] = s.m;
    float f[6];
    weights_to_f32(s.w, f);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      j.w[6 * line + k] = s.w[k];
      j.wf[6 * line + k] = f[k];
    }
  }
  if (j.span) chunk_span(on, signed_offset(m, j.n), line, j.C, j.span);
}

// Generic 1D sweep along dimension DIM: one thread per output cell, taps
// gathered through L1/L2.  Any extents (including n < 6, where the stencil
// wraps more than once).
template <typename T, int DIM>
__global__ void k_advect_generic(const T *__restrict__ fn, T *__restrict__ fnp1, int nx, int ny, int nvx,
                                 int nvy, StencilTable tab) {
  const long long nxy = (long long)nx * ny;
  const long long total = nxy * nvx * nvy;
  const T *__restrict__ w = WeightsOf<T>::get(tab);
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(idx % nx);
    long long r = idx / nx;
    const int iy = (int)(r % ny);
    r /= ny;
    const int ivx = (int)(r % nvx);
    const int ivy = (int)(r / nvx);
    int line, n, i;
    long long stride;
    if (DIM == 0) { line = ivx; n = nx; i = ix; stride = 1; }
    else if (DIM == 1) { line = ivy; n = ny; i = iy; stride = nx; }
    else if (DIM == 2) { line = ix + nx * iy; n = nvx; i = ivx; stride = nxy; }
    else { line = ix + nx * iy; n = nvy; i = ivy; stride = nxy * nvx; }
    const long long base = idx - (long long)i * stride;
    int j = i + tab.m[line];
    if (j >= n) j -= n;
    T tap[6], wl[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      tap[k] = fn[base + (long long)j * stride];
      if (++j == n) j = 0;
    }
    load_weights(w, line, wl);
    fnp1[idx] = interp6(wl, tap[0], tap[1], tap[2], tap[3], tap[4], tap[5]);
  }
}

// Generic fused pair: the tensor product of two 1D stencils (x then y, or
// vx then vy).  out = sum_j wb_j * (sum_k wa_k * f[a+k, b+j]); the inner sum
// is the first sweep, evaluated for the six rows the second sweep needs.
template <typename T, bool V>
__global__ void k_advect_pair_generic(const T *__restrict__ fn, T *__restrict__ fnp1, int nx, int ny, int nvx,
                                      int nvy, StencilTable ta, StencilTable tb) {
  const long long nxy = (long long)nx * ny;
  const long long total = nxy * nvx * nvy;
  const T *__restrict__ wa = WeightsOf<T>::get(ta);
  const T *__restrict__ wb = WeightsOf<T>::get(tb);
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(idx % nx);
    long long r = idx / nx;
    const int iy = (int)(r % ny);
    r /= ny;
    const int ivx = (int)(r % nvx);
    const int ivy = (int)(r / nvx);
    int la, lb, na, nb, ia, ib;
    long long sa, sb;
    if (!V) { la = ivx; lb = ivy; na = nx; nb = ny; ia = ix; ib = iy; sa = 1; sb = nx; }
    else { la = lb = ix + nx * iy; na = nvx; nb = nvy; ia = ivx; ib = ivy; sa = nxy; sb = nxy * nvx; }
    const long long base = idx - (long long)ia * sa - (long long)ib * sb;
    int jb = ib + tb.m[lb];
    if (jb >= nb) jb -= nb;
    const int ja0 = (ia + ta.m[la]) >= na ? ia + ta.m[la] - na : ia + ta.m[la];
    T wla[6], wlb[6], row[6];
    load_weights(wa, la, wla);
    load_weights(wb, lb, wlb);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      int ja = ja0;
      T tap[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        tap[k] = fn[base + (long long)ja * sa + (long long)jb * sb];
        if (++ja == na) ja = 0;
      }
      row[q] = interp6(wla, tap[0], tap[1], tap[2], tap[3], tap[4], tap[5]);
      if (++jb == nb) jb = 0;
    }
    fnp1[idx] = interp6(wlb, row[0], row[1], row[2], row[3], row[4], row[5]);
  }
}

// Slab contexts: vy sweep (after the vx sweep when DVX) of the owned planes,
// one thread per output cell.  Input plane j of the buffer is global plane
// ivy0 - halo + j; output (owned) plane i reads input planes
// i + halo + o + q, q = 0..5, o the column's signed vy offset (the global
// taps (ivy + o + q) mod nvy, which the filled halo makes contiguous).
template <typename T, bool DVX>
__global__ void k_vy_slab_generic(const T *__restrict__ fin, T *__restrict__ fout, int nx, int ny, int nvx,
                                  int nloc, int halo, int nvy_glob, StencilTable tvx, StencilTable tvy,
                                  int *err) {
  const long long nxy = (long long)nx * ny;
  const long long total = nxy * nvx * nloc;
  const long long ystride = nxy * nvx;
  const int nin = nloc + 2 * halo;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long ixy = idx % nxy;
    long long r = idx / nxy;
    const int ivx = (int)(r % nvx);
    const int ivy = (int)(r / nvx);
    int o = tvy.m[ixy];
    if (o > nvy_glob / 2) o -= nvy_glob;
    int j = ivy + halo + o;
    if (j < 0 || j + 5 >= nin) {  // halo too narrow for this column's shift
      atomicOr(err, kErrSlabHalo);
      fout[idx] = T(0);
      continue;
    }
    T wy[6], row[6];
    load_weights(WeightsOf<T>::get(tvy), ixy, wy);
    T wx[6];
    int jx0 = ivx;
    if (DVX) {
      load_weights(WeightsOf<T>::get(tvx), ixy, wx);
      jx0 += tvx.m[ixy];
      if (jx0 >= nvx) jx0 -= nvx;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q, ++j) {
      const T *plane = fin + (long long)j * ystride + ixy;
      if (DVX) {
        T tap[6];
        int jx = jx0;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          tap[k] = plane[(long long)jx * nxy];
          if (++jx == nvx) jx = 0;
        }
        row[q] = interp6(wx, tap[0], tap[1], tap[2], tap[3], tap[4], tap[5]);
      } else {
        row[q] = plane[(long long)ivx * nxy];
      }
    }
    fout[idx] = interp6(wy, row[0], row[1], row[2], row[3], row[4], row[5]);
  }
}

}  // namespace

void free_table(StencilTable &t) {
  cudaFree(t.m);
  cudaFree(t.w);
  cudaFree(t.wf);
  cudaFree(t.span);
  t.m = nullptr;
  t.w = nullptr;
  t.wf = nullptr;
  t.span = nullptr;
  t.span_C = 0;
  t.lines = 0;
  t.valid = false;
}

int alloc_span(StencilTable &t, int C) {
  if (C < 8 || 32 % C) return VLP4D_ERR_UNSUPPORTED;
  // Room for the smallest chunk width, 8 lines.
  if (!t.span) VLP4D_CUDA_TRY(cudaMalloc(&t.span, sizeof(int2) * ((size_t)t.lines / 8 + 1)));
  return VLP4D_OK;
}

int alloc_table(StencilTable &t, int lines, int taps) {
  if (t.m && t.lines >= lines) return VLP4D_OK;
  cudaFree(t.m);
  cudaFree(t.w);
  cudaFree(t.wf);
  cudaFree(t.span);
  t.m = nullptr; t.w = nullptr; t.wf = nullptr;
  t.span = nullptr;
  t.span_C = 0;
  VLP4D_CUDA_TRY(cudaMalloc(&t.m, sizeof(int) * lines));
  VLP4D_CUDA_TRY(cudaMalloc(&t.w, sizeof(double) * taps * lines));
  VLP4D_CUDA_TRY(cudaMalloc(&t.wf, sizeof(float) * taps * lines));
  t.lines = lines;
  t.valid = false;
  return VLP4D_OK;
}

namespace {

int grid_for(long long total, int threads, int sms) {
  long long blocks = (total + threads - 1) / threads;
  const long long cap = (long long)sms * 16;
  return (int)(blocks < cap ? blocks : cap);
}

}  // namespace

// x lines (dim 0) are indexed by ivx with displacement dt*vx; y lines
// (dim 1) by ivy with dt*vy (advection.hpp:113-115, 178-181).  Built on the
// host with the same non-contracted FP64 arithmetic as the device code and
// uploaded; two slots per dimension cache dt/2 and dt of a Strang step.
int ensure_xy_table(vlp4d_ctx *c, int dim, double dt, StencilTable **out, cudaStream_t s) {
  StencilTable *slots = dim == 0 ? c->tab_x : c->tab_y;
  for (int i = 0; i < 2; ++i)
    if (slots[i].valid && slots[i].dt == dt) {
      slots[i].stamp = ++c->table_clock;
      *out = &slots[i];
      return VLP4D_OK;
    }
  // Replace an empty slot, else the least recently used one.
  int pick = !slots[0].valid ? 0 : (!slots[1].valid ? 1 : (slots[0].stamp <= slots[1].stamp ? 0 : 1));
  StencilTable *t = &slots[pick];
  t->valid = false;
  const int vdim = dim == 0 ? 2 : 3;
  const int lines = c->g.n[vdim];
  // Slab contexts hold the vy lines ivy0 .. ivy0 + lines - 1 of the run.
  const int l0 = vdim == 3 ? c->ivy0 : 0;
  int rc = alloc_table(*t, lines);
  if (rc) return rc;
  std::vector<int> hm(lines);
  std::vector<double> hw(6 * (size_t)lines);
  std::vector<float> hwf(6 * (size_t)lines);
  for (int l = 0; l < lines; ++l) {
    const double v = c->g.minp[vdim] + (l0 + l) * c->g.dx[vdim];
    const double disp = dt * v;
    const LineStencil st = line_stencil(disp, c->g.minp[dim], c->g.maxp[dim], c->g.n[dim]);
    hm[l] = st.m;
    float f[6];
    weights_to_f32(st.w, f);
    for (int k = 0; k < 6; ++k) {
      hw[6 * l + k] = st.w[k];
      hwf[6 * l + k] = f[k];
    }
  }
  VLP4D_CUDA_TRY(cudaMemcpyAsync(t->m, hm.data(), sizeof(int) * lines, cudaMemcpyHostToDevice, s));
  VLP4D_CUDA_TRY(cudaMemcpyAsync(t->w, hw.data(), sizeof(double) * 6 * lines, cudaMemcpyHostToDevice, s));
  VLP4D_CUDA_TRY(cudaMemcpyAsync(t->wf, hwf.data(), sizeof(float) * 6 * lines, cudaMemcpyHostToDevice, s));
  // The host vectors die at return; make sure the copies have consumed them.
  VLP4D_CUDA_TRY(cudaStreamSynchronize(s));
  t->dt = dt;
  t->valid = true;
  t->stamp = ++c->table_clock;
  *out = t;
  return VLP4D_OK;
}

void line11(const LineStencil &st, int n, int *m, double W[11], float u[10]) {
  // out[i] = sum_k w_k sum_j w_j f[i + m + k + m + j] = sum_q W_q f[i + 2m + q].
  for (int q = 0; q < 11; ++q) W[q] = 0.;
  for (int k = 0; k < 6; ++k)
    for (int j = 0; j < 6; ++j) W[k + j] += st.w[k] * st.w[j];
  *m = (int)((2LL * st.m) % n);
  // FP32 difference form about tap 5 (the weights sum to one):
  // out = f5 + sum_j u_j (f_{j+1} - f_j), u_j = -(W_0+..+W_j) for j < 5,
  // u_j = W_{j+1}+..+W_10 for j >= 5.
  double acc = 0.;
  for (int j = 0; j < 5; ++j) {
    acc += W[j];
    u[j] = (float)-acc;
  }
  acc = 0.;
  for (int j = 9; j >= 5; --j) {
    acc += W[j + 1];
    u[j] = (float)acc;
  }
}

int build_xy11_table(vlp4d_ctx *c, int dim, double dt, bool transposed, StencilTable &t, cudaStream_t s) {
  t.valid = false;
  const int vdim = dim == 0 ? 2 : 3;
  const int lines = c->g.n[vdim], n = c->g.n[dim];
  const int l0 = vdim == 3 ? c->ivy0 : 0;  // slab contexts: global vy lines
  int rc = alloc_table(t, lines, 11);
  if (rc) return rc;
  std::vector<int> hm(lines);
  std::vector<double> hw(11 * (size_t)lines);
  std::vector<float> hwf(11 * (size_t)lines);
  for (int l = 0; l < lines; ++l) {
    const double v = c->g.minp[vdim] + (l0 + l) * c->g.dx[vdim];
    LineStencil st = line_stencil(dt * v, c->g.minp[dim], c->g.maxp[dim], n);
    if (transposed) st = adjoint_stencil(st, n);
    double W[11];
    float u[10];
    line11(st, n, &hm[l], W, u);
    for (int k = 0; k < 11; ++k) {
      hw[11 * l + k] = W[k];
      hwf[11 * l + k] = k < 10 ? u[k] : 0.f;
    }
  }
  VLP4D_CUDA_TRY(cudaMemcpyAsync(t.m, hm.data(), sizeof(int) * lines, cudaMemcpyHostToDevice, s));
  VLP4D_CUDA_TRY(cudaMemcpyAsync(t.w, hw.data(), sizeof(double) * 11 * lines, cudaMemcpyHostToDevice, s));
  VLP4D_CUDA_TRY(cudaMemcpyAsync(t.wf, hwf.data(), sizeof(float) * 11 * lines, cudaMemcpyHostToDevice, s));
  VLP4D_CUDA_TRY(cudaStreamSynchronize(s));
  t.dt = dt;
  t.valid = true;
  return VLP4D_OK;
}

int ensure_xy11_table(vlp4d_ctx *c, int dim, double dt, StencilTable **out, cudaStream_t s) {
  StencilTable *t = dim == 0 ? &c->tab_x11 : &c->tab_y11;
  if (t->valid && t->dt == dt) {
    *out = t;
    return VLP4D_OK;
  }
  int rc = build_xy11_table(c, dim, dt, false, *t, s);
  if (rc) return rc;
  *out = t;
  return VLP4D_OK;
}

int build_v_tables(vlp4d_ctx *c, double dt, bool vx, bool vy, cudaStream_t s) {
  const int lines = (int)c->g.nxy();
  const int threads = 256, blocks = (lines + threads - 1) / threads;
  VtableJob jobs[2];
  int njobs = 0;
  if (vx) {
    int rc = alloc_table(c->tab_vx, lines);
    if (rc) return rc;
    jobs[njobs++] = {c->ex, c->g.minp[2], c->g.maxp[2], c->g.n[2], c->tab_vx.m, c->tab_vx.w, c->tab_vx.wf, nullptr, 0};
  }
  if (vy) {
    int rc = alloc_table(c->tab_vy, lines);
    if (rc) return rc;
    // With the chunk spans of the v-slab pass when it runs on this shape.
    const int C = vslab_chunk_cols(c);
    c->tab_vy.span_C = 0;
    if (C && threads % 32 == 0 && (rc = alloc_span(c->tab_vy, C)) == VLP4D_OK) c->tab_vy.span_C = C;
    // The vy geometry of the whole run (slab contexts own part of its planes).
    jobs[njobs++] = {c->ey, c->g.minp[3], c->g.maxp[3], c->nvy_glob, c->tab_vy.m, c->tab_vy.w, c->tab_vy.wf,
                     c->tab_vy.span_C ? c->tab_vy.span : nullptr, c->tab_vy.span_C};
  }
  if (!njobs) return VLP4D_OK;
  k_build_vtable<<<dim3((unsigned)blocks, (unsigned)njobs), threads, 0, s>>>(jobs[0], jobs[njobs - 1], lines, dt);
  VLP4D_LAUNCH_CHECK();
  if (vx) c->tab_vx.valid = true;
  if (vy) c->tab_vy.valid = true;
  return VLP4D_OK;
}

int launch_advect_generic(vlp4d_ctx *c, int dim, const void *fn, void *fnp1, const StencilTable *t,
                          cudaStream_t s) {
  const int threads = 256;
  const int blocks = grid_for(c->g.cells(), threads, c->num_sms);
  const int *n = c->g.n;
#define VLP4D_GEN(T, D)                                                                              \
  k_advect_generic<T, D><<<blocks, threads, 0, s>>>((const T *)fn, (T *)fnp1, n[0], n[1], n[2], n[3], *t)
  if (c->dtype == VLP4D_F64) {
    switch (dim) {
      case 0: VLP4D_GEN(double, 0); break;
      case 1: VLP4D_GEN(double, 1); break;
      case 2: VLP4D_GEN(double, 2); break;
      default: VLP4D_GEN(double, 3); break;
    }
  } else {
    switch (dim) {
      case 0: VLP4D_GEN(float, 0); break;
      case 1: VLP4D_GEN(float, 1); break;
      case 2: VLP4D_GEN(float, 2); break;
      default: VLP4D_GEN(float, 3); break;
    }
  }
#undef VLP4D_GEN
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

int launch_advect_pair_generic(vlp4d_ctx *c, bool v, const void *fn, void *fnp1, const StencilTable *ta,
                               const StencilTable *tb, cudaStream_t s) {
  const int threads = 256;
  const int blocks = grid_for(c->g.cells(), threads, c->num_sms);
  const int *n = c->g.n;
  if (c->dtype == VLP4D_F64) {
    if (v) k_advect_pair_generic<double, true><<<blocks, threads, 0, s>>>((const double *)fn, (double *)fnp1, n[0], n[1], n[2], n[3], *ta, *tb);
    else k_advect_pair_generic<double, false><<<blocks, threads, 0, s>>>((const double *)fn, (double *)fnp1, n[0], n[1], n[2], n[3], *ta, *tb);
  } else {
    if (v) k_advect_pair_generic<float, true><<<blocks, threads, 0, s>>>((const float *)fn, (float *)fnp1, n[0], n[1], n[2], n[3], *ta, *tb);
    else k_advect_pair_generic<float, false><<<blocks, threads, 0, s>>>((const float *)fn, (float *)fnp1, n[0], n[1], n[2], n[3], *ta, *tb);
  }
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

int launch_vy_slab_generic(vlp4d_ctx *c, const void *fn_ext, void *fnp1_owned, const StencilTable *tvx,
                           const StencilTable *tvy, cudaStream_t s) {
  const int threads = 256;
  const int blocks = grid_for(c->g.cells(), threads, c->num_sms);
  const int *n = c->g.n;
  StencilTable tx = tvx ? *tvx : StencilTable{};
#define VLP4D_VYS(T, DVX)                                                                                 \
  k_vy_slab_generic<T, DVX><<<blocks, threads, 0, s>>>((const T *)fn_ext, (T *)fnp1_owned, n[0], n[1], n[2], \
                                                      n[3], c->halo, c->nvy_glob, tx, *tvy, c->d_err)
  if (c->dtype == VLP4D_F64) {
    if (tvx) VLP4D_VYS(double, true);
    else VLP4D_VYS(double, false);
  } else {
    if (tvx) VLP4D_VYS(float, true);
    else VLP4D_VYS(float, false);
  }
#undef VLP4D_VYS
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}

}  // namespace vlp4d
