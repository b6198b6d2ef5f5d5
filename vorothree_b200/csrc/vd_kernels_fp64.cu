// vd_kernels_fp64.cu -- the plain FP64 clip kernels.
//
// Compiled with -fmad=false: the reference never fuses a multiply and an
// add, so neither may this path, or its vertices would differ in the last bit
// and the tie-breaking 1e-9 bands could classify differently.
#include "vd_clip.cuh"
#include "vd_internal.h"

namespace vd {

constexpr int kFastWarpsPerBlock = 4;

template <class C, int WPB>
__global__ void __launch_bounds__(WPB * 32) k_clip_fast(const TessDesc T, const WorkList W) {
  extern __shared__ __align__(16) unsigned char smem[];
  WarpPoly<C>* polys = reinterpret_cast<WarpPoly<C>*>(smem);
  clip_worker<C>(T, W, polys[threadIdx.x >> 5]);
}

template <class C>
__global__ void __launch_bounds__(128) k_clip_big(const TessDesc T, const WorkList W, WarpPoly<C>* scratch) {
  const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  clip_worker<C>(T, W, scratch[gw]);
}

static_assert(sizeof(WarpPoly<FastCfg>) == sizeof(WarpPoly<FastCfgCount>), "same layout");

cudaError_t clip_fp64_info(ClipLaunchInfo* info) {
  info->smem_per_warp = sizeof(WarpPoly<FastCfg>);
  info->warps_per_block = kFastWarpsPerBlock;
  info->big_scratch_per_warp = sizeof(WarpPoly<BigCfg>);
  const size_t smem = sizeof(WarpPoly<FastCfg>) * kFastWarpsPerBlock;
  cudaError_t e = cudaFuncSetAttribute(k_clip_fast<FastCfg, kFastWarpsPerBlock>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_clip_fast<FastCfgCount, kFastWarpsPerBlock>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int nb = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_clip_fast<FastCfg, kFastWarpsPerBlock>,
                                                    kFastWarpsPerBlock * 32, smem);
  info->blocks_per_sm = nb;
  return e;
}

cudaError_t launch_clip_fp64_fast(const TessDesc& T, const WorkList& W, int nblocks, bool count,
                                  cudaStream_t s) {
  const size_t smem = sizeof(WarpPoly<FastCfg>) * kFastWarpsPerBlock;
  if (count)
    k_clip_fast<FastCfgCount, kFastWarpsPerBlock><<<nblocks, kFastWarpsPerBlock * 32, smem, s>>>(T, W);
  else
    k_clip_fast<FastCfg, kFastWarpsPerBlock><<<nblocks, kFastWarpsPerBlock * 32, smem, s>>>(T, W);
  return cudaGetLastError();
}

cudaError_t launch_clip_fp64_big(const TessDesc& T, const WorkList& W, void* scratch, int nwarps,
                                 cudaStream_t s) {
  const int nblocks = nwarps / 4;  // the caller sizes scratch for whole blocks of 4 warps
  k_clip_big<BigCfg><<<nblocks, 128, 0, s>>>(T, W, reinterpret_cast<WarpPoly<BigCfg>*>(scratch));
  return cudaGetLastError();
}

}  // namespace vd
