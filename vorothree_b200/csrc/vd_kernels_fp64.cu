// vd_kernels_fp64.cu -- the plain FP64 clip kernels.
//
// Compiled with -fmad=false: the reference never fuses a multiply and an
// add, so neither may this path, or its vertices would differ in the last bit
// and the tie-breaking 1e-9 bands could classify differently.
#include "vd_clip.cuh"
#include "vd_clip_hub.cuh"
#include "vd_internal.h"

namespace vd {


// shared memory admits 7 blocks of 4 warps per SM; keep registers in step
// (without the bound ptxas takes ~100 registers and only 4 blocks fit)
constexpr int kFp64MinBlocks = 7;
// the batched kernel (member lookup, descriptors in device memory) needs
// more registers: measured fastest at 5 blocks (96 registers; 7 blocks:
// -13%, 6: -12%, 4: -9%)
constexpr int kBatchMinBlocks = 5;

cudaError_t clip_fp64_info(ClipLaunchInfo* info) {
  info->smem_per_warp = sizeof(WarpPoly<FastCfg>);
  info->warps_per_block = kFastWarpsPerBlock;
  info->big_scratch_per_warp = sizeof(WarpPoly<BigCfg>);
  const size_t smem = sizeof(WarpPoly<FastCfg>) * kFastWarpsPerBlock;
  const size_t smemc = sizeof(WarpPoly<FastCfgCount>) * kFastWarpsPerBlock;
  cudaError_t e = cudaFuncSetAttribute(k_clip_fast<FastCfg, kFastWarpsPerBlock, kFp64MinBlocks>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_clip_fast<FastCfgCount, kFastWarpsPerBlock, kFp64MinBlocks>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemc);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_clip_fast<FastCfg, kFastWarpsPerBlock, kFp64MinBlocks, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int nb = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_clip_fast<FastCfg, kFastWarpsPerBlock, kFp64MinBlocks>,
                                                    kFastWarpsPerBlock * 32, smem);
  info->blocks_per_sm = nb;
  return e;
}

cudaError_t launch_clip_fp64_fast(const TessDesc& T, const WorkList& W, int nblocks, bool count,
                                  cudaStream_t s, bool noop) {
  const size_t smem = sizeof(WarpPoly<FastCfg>) * kFastWarpsPerBlock;
  const size_t smemc = sizeof(WarpPoly<FastCfgCount>) * kFastWarpsPerBlock;
  if (count)
    k_clip_fast<FastCfgCount, kFastWarpsPerBlock, kFp64MinBlocks><<<nblocks, kFastWarpsPerBlock * 32, smemc, s>>>(T, W);
  else if (noop)
    k_clip_fast<FastCfg, kFastWarpsPerBlock, kFp64MinBlocks, true><<<nblocks, kFastWarpsPerBlock * 32, smem, s>>>(T, W);
  else
    k_clip_fast<FastCfg, kFastWarpsPerBlock, kFp64MinBlocks><<<nblocks, kFastWarpsPerBlock * 32, smem, s>>>(T, W);
  return cudaGetLastError();
}

cudaError_t launch_clip_fp64_big(const TessDesc& T, const WorkList& W, void* scratch, int nwarps,
                                 cudaStream_t s, bool noop) {
  const int nblocks = nwarps / 4;  // the caller sizes scratch for whole blocks of 4 warps
  if (noop)
    k_clip_big<BigCfg, true><<<nblocks, 128, 0, s>>>(T, W, reinterpret_cast<WarpPoly<BigCfg>*>(scratch));
  else
    k_clip_big<BigCfg><<<nblocks, 128, 0, s>>>(T, W, reinterpret_cast<WarpPoly<BigCfg>*>(scratch));
  return cudaGetLastError();
}

// the huge tier's scratch: a polytope per block
size_t clip_huge_scratch_per_block() { return sizeof(WarpPoly<HugeCfg>); }

// the huge kernels' dynamic shared memory (the slot layout's per-clip state,
// above the 48 KB a kernel gets without asking)
template <class K>
static cudaError_t huge_smem(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t launch_clip_fp64_huge(const TessDesc& T, const WorkList& W, void* scratch, int nblocks, bool narrow,
                                  cudaStream_t s) {
  WarpPoly<HugeCfg>* polys = reinterpret_cast<WarpPoly<HugeCfg>*>(scratch);
  if (narrow) {
    constexpr size_t sm = sizeof(HubShared<kHugeBlockWarpsNarrow>);
    cudaError_t e = huge_smem(k_clip_huge_block<HugeCfg, kHugeBlockWarpsNarrow>, sm);
    if (e != cudaSuccess) return e;
    k_clip_huge_block<HugeCfg, kHugeBlockWarpsNarrow><<<nblocks, kHugeBlockWarpsNarrow * 32, sm, s>>>(T, W, polys);
  } else {
    constexpr size_t sm = sizeof(HubShared<kHugeBlockWarps>);
    cudaError_t e = huge_smem(k_clip_huge_block<HugeCfg, kHugeBlockWarps>, sm);
    if (e != cudaSuccess) return e;
    k_clip_huge_block<HugeCfg, kHugeBlockWarps><<<nblocks, kHugeBlockWarps * 32, sm, s>>>(T, W, polys);
  }
  return cudaGetLastError();
}

cudaError_t launch_clip_fp64_huge_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess,
                                          const WorkList& W, void* scratch, int nblocks, cudaStream_t s) {
  WarpPoly<HugeCfg>* polys = reinterpret_cast<WarpPoly<HugeCfg>*>(scratch);
  // (16-warp blocks: the width that wins on the slot layout)
  constexpr size_t sm = sizeof(HubShared<kHugeBlockWarpsNarrow>);
  cudaError_t e = huge_smem(k_clip_huge_block_batched<HugeCfg, kHugeBlockWarpsNarrow>, sm);
  if (e != cudaSuccess) return e;
  k_clip_huge_block_batched<HugeCfg, kHugeBlockWarpsNarrow>
      <<<nblocks, kHugeBlockWarpsNarrow * 32, sm, s>>>(descs, tess_off, ntess, W, polys);
  return cudaGetLastError();
}

cudaError_t launch_clip_fp64_fast_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess,
                                          const WorkList& W, int nblocks, bool count, cudaStream_t s) {
  const size_t smem = sizeof(WarpPoly<FastCfg>) * kFastWarpsPerBlock;
  const size_t smemc = sizeof(WarpPoly<FastCfgCount>) * kFastWarpsPerBlock;
  if (count)
    k_clip_fast_batched<FastCfgCount, kFastWarpsPerBlock, kBatchMinBlocks>
        <<<nblocks, kFastWarpsPerBlock * 32, smemc, s>>>(descs, tess_off, ntess, W);
  else
    k_clip_fast_batched<FastCfg, kFastWarpsPerBlock, kBatchMinBlocks>
        <<<nblocks, kFastWarpsPerBlock * 32, smem, s>>>(descs, tess_off, ntess, W);
  return cudaGetLastError();
}

cudaError_t launch_clip_fp64_big_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess,
                                         const WorkList& W, void* scratch, int nwarps, cudaStream_t s) {
  k_clip_big_batched<BigCfg><<<nwarps / 4, 128, 0, s>>>(descs, tess_off, ntess, W,
                                                       reinterpret_cast<WarpPoly<BigCfg>*>(scratch));
  return cudaGetLastError();
}

cudaError_t clip_fp64_batched_setup(int* blocks_per_sm) {
  const size_t smem = sizeof(WarpPoly<FastCfg>) * kFastWarpsPerBlock;
  const size_t smemc = sizeof(WarpPoly<FastCfgCount>) * kFastWarpsPerBlock;
  cudaError_t e = cudaFuncSetAttribute(k_clip_fast_batched<FastCfg, kFastWarpsPerBlock, kBatchMinBlocks>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_clip_fast_batched<FastCfgCount, kFastWarpsPerBlock, kBatchMinBlocks>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemc);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      blocks_per_sm, k_clip_fast_batched<FastCfg, kFastWarpsPerBlock, kBatchMinBlocks>, kFastWarpsPerBlock * 32, smem);
}

constexpr int kMedWarpsPerBlock = 2;

cudaError_t clip_med_setup(ClipLaunchInfo* info) {
  const size_t smem = sizeof(WarpPoly<MedCfg>) * kMedWarpsPerBlock;
  info->smem_per_warp = sizeof(WarpPoly<MedCfg>);
  info->warps_per_block = kMedWarpsPerBlock;
  cudaError_t e = cudaFuncSetAttribute(k_clip_fast<MedCfg, kMedWarpsPerBlock, 1>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  static_assert(sizeof(WarpPoly<MedCfgNC>) <= sizeof(WarpPoly<MedCfg>), "one shared-memory size serves both");
  e = cudaFuncSetAttribute(k_clip_fast<MedCfgNC, kMedWarpsPerBlock, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_clip_fast<MedCfgNC, kMedWarpsPerBlock, 1, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_clip_fast_batched<MedCfg, kMedWarpsPerBlock, 1>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int nb = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_clip_fast<MedCfg, kMedWarpsPerBlock, 1>,
                                                    kMedWarpsPerBlock * 32, smem);
  info->blocks_per_sm = nb;
  return e;
}

cudaError_t launch_clip_med(const TessDesc& T, const WorkList& W, int nblocks, bool count, cudaStream_t s,
                            bool noop) {
  const size_t smem = sizeof(WarpPoly<MedCfg>) * kMedWarpsPerBlock;
  if (count)
    k_clip_fast<MedCfg, kMedWarpsPerBlock, 1><<<nblocks, kMedWarpsPerBlock * 32, smem, s>>>(T, W);
  else if (noop)
    k_clip_fast<MedCfgNC, kMedWarpsPerBlock, 1, true><<<nblocks, kMedWarpsPerBlock * 32, smem, s>>>(T, W);
  else
    k_clip_fast<MedCfgNC, kMedWarpsPerBlock, 1><<<nblocks, kMedWarpsPerBlock * 32, smem, s>>>(T, W);
  return cudaGetLastError();
}

cudaError_t launch_clip_med_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess,
                                    const WorkList& W, int nblocks, cudaStream_t s) {
  const size_t smem = sizeof(WarpPoly<MedCfg>) * kMedWarpsPerBlock;
  k_clip_fast_batched<MedCfg, kMedWarpsPerBlock, 1>
      <<<nblocks, kMedWarpsPerBlock * 32, smem, s>>>(descs, tess_off, ntess, W);
  return cudaGetLastError();
}

}  // namespace vd
