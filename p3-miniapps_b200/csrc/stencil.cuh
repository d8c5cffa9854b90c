// Six-tap interpolation of one output from its stencil taps, and the
// per-line weight loads shared by the advection kernels.
//
// FP64 (the reference's arithmetic, advection.hpp:128-135): out = sum_k w_k f_k.
// FP32 storage, adjacent-difference form:
//   out = f_2 + sum_{j=0..4} v_j (f_{j+1} - f_j),
//   v = (-w0, -(w0+w1), w3+w4+w5, w4+w5, w5)   (from the FP64 weights),
// equal to the plain form in exact arithmetic because the weights sum to one.
// In FP32 it makes every rounding term (weights, products, partial sums)
// proportional to the local variation of f instead of to f itself: with the
// plain form the FP32-rounded weights of a line are re-applied identically
// every step and their bias accumulates in the field energy.  Neighbouring
// outputs share their differences, which the fused kernels exploit.
#pragma once

#include "internal.cuh"

namespace vlp4d {

__device__ __forceinline__ double interp6(const double (&w)[6], double f0, double f1, double f2, double f3,
                                          double f4, double f5) {
  double acc = w[0] * f0;
  acc = fma(w[1], f1, acc);
  acc = fma(w[2], f2, acc);
  acc = fma(w[3], f3, acc);
  acc = fma(w[4], f4, acc);
  acc = fma(w[5], f5, acc);
  return acc;
}

// The adjacent-difference form on precomputed differences d_j = f_{j+1} - f_j.
__device__ __forceinline__ float interp_diff(const float (&v)[6], float f2, float d0, float d1, float d2, float d3,
                                             float d4) {
  float acc = v[0] * d0;
  acc = fmaf(v[1], d1, acc);
  acc = fmaf(v[2], d2, acc);
  acc = fmaf(v[3], d3, acc);
  acc = fmaf(v[4], d4, acc);
  return f2 + acc;
}

// v holds the difference weights in slots 0..4.
__device__ __forceinline__ float interp6(const float (&v)[6], float f0, float f1, float f2, float f3, float f4,
                                         float f5) {
  return interp_diff(v, f2, f1 - f0, f2 - f1, f3 - f2, f4 - f3, f5 - f4);
}

// Packed FP32 pairs (the sm_100 f32x2 FMA/MUL/ADD instructions).  Each lane
// rounds exactly as the scalar round-to-nearest operation does, so the
// packed evaluation of the difference form gives the same bits as the
// scalar one.  a - b is formed as fma(b, -1, a): -b is exact, so the single
// rounding is that of the subtraction.
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

// interp_diff on two lanes that share their weights; v[j] = (v_j, v_j).
__device__ __forceinline__ float2 interp_diff2(const float2 (&v)[5], float2 f2, float2 d0, float2 d1, float2 d2,
                                               float2 d3, float2 d4) {
  float2 acc = __fmul2_rn(v[0], d0);
  acc = __ffma2_rn(v[1], d1, acc);
  acc = __ffma2_rn(v[2], d2, acc);
  acc = __ffma2_rn(v[3], d3, acc);
  acc = __ffma2_rn(v[4], d4, acc);
  return __fadd2_rn(f2, acc);
}

// Weights as the sweeps consume them: the six FP64 weights, or the five FP32
// difference weights duplicated into both lanes of a pair.
template <typename T>
struct SweepW {
  T w[6];
};
template <>
struct SweepW<float> {
  float2 v[5];
};
__device__ __forceinline__ void make_sweep_w(const double (&w)[6], SweepW<double> &s) {
#pragma unroll
  for (int k = 0; k < 6; ++k) s.w[k] = w[k];
}
__device__ __forceinline__ void make_sweep_w(const float (&w)[6], SweepW<float> &s) {
#pragma unroll
  for (int k = 0; k < 5; ++k) s.v[k] = make_float2(w[k], w[k]);
}

// Four x-swept outputs from the twelve staged values t[0..11] starting at the
// aligned column a0 = c0 + mx - r; output q uses t[r+q .. r+q+5].  r is the
// same for the whole CTA (c0 is a multiple of 4), so the switch is uniform.
template <int R_>
__device__ __forceinline__ void x4_from(const double (&t)[12], const SweepW<double> &w, double (&o)[4]) {
#pragma unroll
  for (int q = 0; q < 4; ++q)
    o[q] = interp6(w.w, t[R_ + q], t[R_ + q + 1], t[R_ + q + 2], t[R_ + q + 3], t[R_ + q + 4], t[R_ + q + 5]);
}
// FP32: outputs (0,1) and (2,3) as packed pairs; pair j of differences is
// (d_j, d_{j+1}) with d_j = t[r+j+1] - t[r+j].
template <int R_>
__device__ __forceinline__ void x4_from(const float (&t)[12], const SweepW<float> &w, float (&o)[4]) {
  float d[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) d[j] = t[R_ + j + 1] - t[R_ + j];
  float2 dp[7];
#pragma unroll
  for (int j = 0; j < 7; ++j) dp[j] = make_float2(d[j], d[j + 1]);
  const float2 lo = interp_diff2(w.v, make_float2(t[R_ + 2], t[R_ + 3]), dp[0], dp[1], dp[2], dp[3], dp[4]);
  const float2 hi = interp_diff2(w.v, make_float2(t[R_ + 4], t[R_ + 5]), dp[2], dp[3], dp[4], dp[5], dp[6]);
  o[0] = lo.x;
  o[1] = lo.y;
  o[2] = hi.x;
  o[3] = hi.y;
}
template <typename T>
__device__ __forceinline__ void sweep_x4(const T (&t)[12], int r, const SweepW<T> &w, T (&o)[4]) {
  switch (r) {
    case 0: x4_from<0>(t, w, o); break;
    case 1: x4_from<1>(t, w, o); break;
    case 2: x4_from<2>(t, w, o); break;
    default: x4_from<3>(t, w, o); break;
  }
}

template <typename T>
struct WeightsOf;
template <>
struct WeightsOf<double> {
  static __device__ __forceinline__ const double *get(const StencilTable &t) { return t.w; }
};
template <>
struct WeightsOf<float> {
  static __device__ __forceinline__ const float *get(const StencilTable &t) { return t.wf; }
};

template <typename T>
__device__ __forceinline__ void load_weights(const T *__restrict__ w, long long line, T (&out)[6]) {
#pragma unroll
  for (int k = 0; k < 6; ++k) out[k] = __ldg(w + 6 * line + k);
}

}  // namespace vlp4d
