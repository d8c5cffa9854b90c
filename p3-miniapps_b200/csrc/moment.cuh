// Second stage of the velocity moment (field_rho, miniapps/vlp4d/thrust/
// field.cpp:6-32): rho[ixy] = dvx * dvy * (sum over the plane groups of the
// FP64 partial sums part[group][ixy]).
//
// The groups are added in a fixed order that does not depend on the launch
// shape: kMomentSlices contiguous ranges of groups, [s*G/S, (s+1)*G/S), each
// summed in increasing group order, then the slices in increasing order.
// Blocks of 32 cells x kMomentSlices slices sum the slices of a cell in
// parallel (the partials of small grids are few cells of many groups; one
// thread per cell left most of the GPU idle and the kernel bound by the
// latency of its sequential loads).
#pragma once

namespace vlp4d {

constexpr int kMomentSlices = 16;
constexpr int kMomentCells = 32;  // cells per block; blockDim = kMomentCells x kMomentSlices

__device__ __forceinline__ void moment_finish(const double *__restrict__ part, double *__restrict__ rho,
                                              long long nxy, int groups, double dvx, double dvy) {
  __shared__ double sl[kMomentSlices][kMomentCells];
  const int cx = threadIdx.x % kMomentCells, s = threadIdx.x / kMomentCells;
  const long long ixy = (long long)blockIdx.x * kMomentCells + cx;
  const int g0 = (int)((long long)groups * s / kMomentSlices);
  const int g1 = (int)((long long)groups * (s + 1) / kMomentSlices);
  double acc = 0.0;
  if (ixy < nxy) {
    int g = g0;
    // Loads of eight groups issued before their adds (fixed order).
    for (; g + 8 <= g1; g += 8) {
      double v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = part[(long long)(g + k) * nxy + ixy];
#pragma unroll
      for (int k = 0; k < 8; ++k) acc += v[k];
    }
    for (; g < g1; ++g) acc += part[(long long)g * nxy + ixy];
  }
  sl[s][cx] = acc;
  __syncthreads();
  if (s == 0 && ixy < nxy) {
    double sum = 0.0;
#pragma unroll
    for (int k = 0; k < kMomentSlices; ++k) sum += sl[k][cx];
    rho[ixy] = sum * dvx * dvy;  // field.cpp:23 (sum * dvx * dvy)
  }
}

}  // namespace vlp4d
