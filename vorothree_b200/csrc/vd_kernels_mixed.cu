// vd_kernels_mixed.cu -- mixed-precision clip kernels (not built yet).
#include "vd_internal.h"

namespace vd {

cudaError_t clip_mixed_info(ClipLaunchInfo* info) {
  *info = ClipLaunchInfo{0, 1, 0, 0};
  return cudaSuccess;
}

cudaError_t launch_clip_mixed_fast(const TessDesc&, const WorkList&, int, bool, cudaStream_t) {
  return cudaErrorNotSupported;
}

}  // namespace vd
