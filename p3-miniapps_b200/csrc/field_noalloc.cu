// field_rho without any device allocation: vlp4d_field_rho_noalloc.
//
// Who needs it: callers that cannot call cudaMalloc/cudaFree on their path,
// for instance a host application whose device memory is entirely handed to
// its own pool allocator, or a time loop that must not pay cudaFree's
// device-wide synchronisation.  vlp4d_ctx_create allocates the context's
// scratch with cudaMalloc, so such callers use this entry point instead of
// vlp4d_field_rho: they pass f and the output rho; the partial sums of the
// two-level reduction live in a fixed array compiled into this library.
//
// The scratch is g_rho_scratch below: kNoallocScratchDoubles FP64 values
// (4 MiB) on every GPU that loads the library, held until the process exits.
// It bounds nx*ny to kNoallocScratchDoubles.  Every call on a device shares
// it: two calls whose kernels overlap on the GPU (different streams, or
// different host threads) race on it, so callers serialise them (one stream,
// or their own ordering).  Each call writes every partial it later reads, so
// nothing needs clearing between calls and the contents left by the last
// call do not matter.
//
// Host code cannot pass `g_rho_scratch` to a kernel: in host code the name
// is a host-side stand-in, not a device address.  The first call on each
// device, with that device current, looks the address up once with
// cudaGetSymbolAddress and caches it for the life of the process; that
// first call should come before any stream capture on that device.  The
// cache assumes the device's primary context lives as long as the process:
// after cudaDeviceReset (or anything else that destroys the primary context
// and reloads this module) the cached address is stale, so such callers
// must not use this entry point after a reset.
#include <mutex>

#include "internal.cuh"
#include "moment.cuh"

namespace vlp4d {

constexpr long long kNoallocScratchDoubles = 1LL << 19;  // 4 MiB of FP64 partial sums

static __device__ __align__(256) double g_rho_scratch[kNoallocScratchDoubles];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double *g_scratch_ptr[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};

// One-time, per-device lookup of the scratch array's device address (the
// current device must be `dev`).
int noalloc_setup(int dev, double **ptr, int *sms) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_rho_scratch);
    if (e != cudaSuccess) {
      set_error(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
      return VLP4D_ERR_CUDA;
    }
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
      set_error(std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
      return VLP4D_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<double *>(p);
    g_sms[dev] = n;
  }
  *ptr = g_scratch_ptr[dev];
  *sms = g_sms[dev];
  return VLP4D_OK;
}

// Same two-level, fixed-order reduction as field_rho: block (column chunk,
// plane group) -> partial[group][ixy]; then rho = (sum of groups) * dvx * dvy.
template <typename T>
__global__ void k_noalloc_rho_partial(const T *__restrict__ f, double *__restrict__ part, long long nxy,
                                      long long nv, int groups) {
  const long long ixy = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int g = blockIdx.y;
  if (ixy >= nxy) return;
  const long long v0 = nv * g / groups, v1 = nv * (g + 1) / groups;
  double s = 0.0;
  const T *p = f + ixy + v0 * nxy;
#pragma unroll 8
  for (long long v = v0; v < v1; ++v, p += nxy) s += (double)__ldg(p);
  part[(long long)g * nxy + ixy] = s;
}

// The same fixed-order second stage as the context's (moment.cuh).
__global__ void __launch_bounds__(kMomentCells * kMomentSlices)
    k_noalloc_rho_finish(const double *__restrict__ part, double *__restrict__ rho, long long nxy, int groups,
                         double dvx, double dvy) {
  moment_finish(part, rho, nxy, groups, dvx, dvy);
}

}  // namespace
}  // namespace vlp4d

using namespace vlp4d;

extern "C" int vlp4d_field_rho_noalloc(const void *fn, int dtype, int nx, int ny, int nvx, int nvy, double dvx,
                                       double dvy, double *rho, void *stream) {
  if (!fn || !rho) {
    set_error("field_rho_noalloc: NULL buffer");
    return VLP4D_ERR_INVALID_ARG;
  }
  if (dtype != VLP4D_F64 && dtype != VLP4D_F32) {
    set_error("field_rho_noalloc: dtype must be VLP4D_F64 or VLP4D_F32");
    return VLP4D_ERR_INVALID_ARG;
  }
  if (nx < 1 || ny < 1 || nvx < 1 || nvy < 1) {
    set_error("field_rho_noalloc: extents must be positive");
    return VLP4D_ERR_INVALID_ARG;
  }
  const long long nxy = (long long)nx * ny, nv = (long long)nvx * nvy;
  if (nxy > kNoallocScratchDoubles) {
    set_error("field_rho_noalloc: nx*ny = " + std::to_string(nxy) + " exceeds the built-in scratch of " +
              std::to_string(kNoallocScratchDoubles) + " values; use vlp4d_field_rho with a context");
    return VLP4D_ERR_INVALID_ARG;
  }
  int dev = 0;
  VLP4D_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("field_rho_noalloc: device index out of range");
    return VLP4D_ERR_UNSUPPORTED;
  }
  double *part = nullptr;
  int sms = 0;
  int rc = noalloc_setup(dev, &part, &sms);
  if (rc) return rc;
  // Same group count as a context would choose, limited by the scratch.
  long long groups = ((long long)sms * 8 * 256 + nxy - 1) / nxy;
  if (groups > nv) groups = nv;
  if (groups > 1024) groups = 1024;
  if (groups > kNoallocScratchDoubles / nxy) groups = kNoallocScratchDoubles / nxy;
  if (groups < 1) groups = 1;
  const int threads = 256;
  cudaStream_t s = (cudaStream_t)stream;
  dim3 grid((unsigned)((nxy + threads - 1) / threads), (unsigned)groups);
  if (dtype == VLP4D_F64)
    k_noalloc_rho_partial<double><<<grid, threads, 0, s>>>((const double *)fn, part, nxy, nv, (int)groups);
  else
    k_noalloc_rho_partial<float><<<grid, threads, 0, s>>>((const float *)fn, part, nxy, nv, (int)groups);
  VLP4D_LAUNCH_CHECK();
  k_noalloc_rho_finish<<<(unsigned)((nxy + kMomentCells - 1) / kMomentCells), kMomentCells * kMomentSlices, 0, s>>>(
      part, rho, nxy, (int)groups, dvx, dvy);
  VLP4D_LAUNCH_CHECK();
  return VLP4D_OK;
}
