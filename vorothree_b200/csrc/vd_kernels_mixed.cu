// vd_kernels_mixed.cu -- the mixed-precision clip kernels.
//
// Vertex classification runs in FP32 on generator-relative coordinates under
// a static forward error bound; vertices near the +-1e-9 thresholds fall back
// to the plain path's FP64 formula, so every decision equals the FP64
// path's.  Vertex construction and all reductions stay FP64.  Like the plain
// path, this translation unit is compiled with -fmad=false (the FP32
// classification uses explicit fmaf), so results equal the plain path's bit
// for bit.
#include "vd_clip.cuh"
#include "vd_internal.h"

namespace vd {


// 5 blocks of 4 warps per SM: the mixed kernel needs more registers than
// the plain one (FP32 copies and the error bound); measured fastest at 5
// (7 blocks: -12%, 6: -11%, 4: -6%)
constexpr int kMixedMinBlocks = 5;

cudaError_t clip_mixed_info(ClipLaunchInfo* info) {
  info->smem_per_warp = sizeof(WarpPoly<MixedCfg>);
  info->warps_per_block = kFastWarpsPerBlock;
  info->big_scratch_per_warp = sizeof(WarpPoly<BigCfg>);
  const size_t smem = sizeof(WarpPoly<MixedCfg>) * kFastWarpsPerBlock;
  const size_t smemc = sizeof(WarpPoly<MixedCfgCount>) * kFastWarpsPerBlock;
  cudaError_t e = cudaFuncSetAttribute(k_clip_fast<MixedCfg, kFastWarpsPerBlock, kMixedMinBlocks>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_clip_fast<MixedCfgCount, kFastWarpsPerBlock, kMixedMinBlocks>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemc);
  if (e != cudaSuccess) return e;
  int nb = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_clip_fast<MixedCfg, kFastWarpsPerBlock, kMixedMinBlocks>,
                                                    kFastWarpsPerBlock * 32, smem);
  info->blocks_per_sm = nb;
  return e;
}

cudaError_t launch_clip_mixed_fast(const TessDesc& T, const WorkList& W, int nblocks, bool count,
                                   cudaStream_t s) {
  const size_t smem = sizeof(WarpPoly<MixedCfg>) * kFastWarpsPerBlock;
  const size_t smemc = sizeof(WarpPoly<MixedCfgCount>) * kFastWarpsPerBlock;
  if (count)
    k_clip_fast<MixedCfgCount, kFastWarpsPerBlock, kMixedMinBlocks><<<nblocks, kFastWarpsPerBlock * 32, smemc, s>>>(T, W);
  else
    k_clip_fast<MixedCfg, kFastWarpsPerBlock, kMixedMinBlocks><<<nblocks, kFastWarpsPerBlock * 32, smem, s>>>(T, W);
  return cudaGetLastError();
}

cudaError_t launch_clip_mixed_fast_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess,
                                           const WorkList& W, int nblocks, bool count, cudaStream_t s) {
  const size_t smem = sizeof(WarpPoly<MixedCfg>) * kFastWarpsPerBlock;
  const size_t smemc = sizeof(WarpPoly<MixedCfgCount>) * kFastWarpsPerBlock;
  if (count)
    k_clip_fast_batched<MixedCfgCount, kFastWarpsPerBlock, kMixedMinBlocks>
        <<<nblocks, kFastWarpsPerBlock * 32, smemc, s>>>(descs, tess_off, ntess, W);
  else
    k_clip_fast_batched<MixedCfg, kFastWarpsPerBlock, kMixedMinBlocks>
        <<<nblocks, kFastWarpsPerBlock * 32, smem, s>>>(descs, tess_off, ntess, W);
  return cudaGetLastError();
}

cudaError_t clip_mixed_batched_setup(int* blocks_per_sm) {
  const size_t smem = sizeof(WarpPoly<MixedCfg>) * kFastWarpsPerBlock;
  const size_t smemc = sizeof(WarpPoly<MixedCfgCount>) * kFastWarpsPerBlock;
  cudaError_t e = cudaFuncSetAttribute(k_clip_fast_batched<MixedCfg, kFastWarpsPerBlock, kMixedMinBlocks>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_clip_fast_batched<MixedCfgCount, kFastWarpsPerBlock, kMixedMinBlocks>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemc);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      blocks_per_sm, k_clip_fast_batched<MixedCfg, kFastWarpsPerBlock, kMixedMinBlocks>, kFastWarpsPerBlock * 32, smem);
}

}  // namespace vd
