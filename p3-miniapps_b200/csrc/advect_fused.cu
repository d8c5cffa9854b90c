// Bandwidth-optimised fused advection kernels (x/y plane pass and v-slab
// pass).  Placeholder dispatch: every shape currently uses the generic
// kernels of advect.cu.
#include "internal.cuh"

namespace vlp4d {

bool xy_fused_supported(const vlp4d_ctx *) { return false; }
bool vv_fused_supported(const vlp4d_ctx *) { return false; }

int launch_advect_xy(vlp4d_ctx *, const void *, void *, const StencilTable *, const StencilTable *, bool, bool,
                     bool, cudaStream_t) {
  set_error("fused x/y pass not available for this shape");
  return VLP4D_ERR_UNSUPPORTED;
}

int launch_advect_vxvy(vlp4d_ctx *, const void *, void *, bool, bool, cudaStream_t) {
  set_error("fused vx/vy pass not available for this shape");
  return VLP4D_ERR_UNSUPPORTED;
}

}  // namespace vlp4d
