// Six-tap interpolation of one output from its stencil taps, and the
// per-line weight loads shared by the advection kernels.
//
// FP64 (the reference's arithmetic, advection.hpp:128-135): out = sum_k w_k f_k.
// FP32 storage: out = f_2 + sum_{k != 2} w_k (f_k - f_2).  The two are equal in
// exact arithmetic because the weights sum to one.  In FP32 the difference
// form makes every rounding term (weights, products, partial sums)
// proportional to the local variation of f instead of to f itself; with the
// plain form, the FP32-rounded weights of a line are re-applied identically
// every step and their bias accumulates in the field energy.
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

__device__ __forceinline__ float interp6(const float (&w)[6], float f0, float f1, float f2, float f3, float f4,
                                         float f5) {
  float acc = w[0] * (f0 - f2);
  acc = fmaf(w[1], f1 - f2, acc);
  acc = fmaf(w[3], f3 - f2, acc);
  acc = fmaf(w[4], f4 - f2, acc);
  acc = fmaf(w[5], f5 - f2, acc);
  return f2 + acc;
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
