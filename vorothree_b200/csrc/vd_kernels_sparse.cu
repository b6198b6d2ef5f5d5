// vd_kernels_sparse.cu -- the shared-memory tier on the slot layout
// (vd_clip_sparse.cuh): plain FP64 and mixed-precision classification,
// single tessellations and batches.
//
// Compiled with -fmad=false like every FP64 path: the reference never fuses
// a multiply and an add, so neither may this one.
#include "vd_clip_sparse.cuh"
#include "vd_internal.h"

namespace vd {

// blocks of 4 warps per SM the register budget must admit (shared memory
// admits this many too): single tessellations are compiled for 5, 6 and 7
// (a tuning setting, 7 by default: 1 M uniform cells 32.5 ms against 33.5 at
// 6 and 33.7 at 5; 8 spills more and was slower; the instrumented variant for
// 6 only), batches for 6 (the 4096-member batch: 30.1 M cells/s against
// 29.4 M at 7, whose member lookup spills more)
constexpr int kSparseBatchMinBlocks = 6;

namespace {

template <class C, int MINB, bool NOOP = false>
cudaError_t setup_one(ClipLaunchInfo* info) {
  const size_t smem = sizeof(SparsePoly<C>) * kFastWarpsPerBlock;
  cudaError_t e = cudaFuncSetAttribute(k_clip_sparse<C, kFastWarpsPerBlock, MINB, NOOP>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess || !info) return e;
  info->smem_per_warp = sizeof(SparsePoly<C>);
  info->warps_per_block = kFastWarpsPerBlock;
  info->big_scratch_per_warp = 0;
  int nb = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_clip_sparse<C, kFastWarpsPerBlock, MINB, NOOP>,
                                                    kFastWarpsPerBlock * 32, smem);
  info->blocks_per_sm = nb;
  return e;
}

template <class C, int MINB>
cudaError_t setup_batched(int* blocks_per_sm) {
  const size_t smem = sizeof(SparsePoly<C>) * kFastWarpsPerBlock;
  cudaError_t e = cudaFuncSetAttribute(k_clip_sparse_batched<C, kFastWarpsPerBlock, MINB>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess || !blocks_per_sm) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      blocks_per_sm, k_clip_sparse_batched<C, kFastWarpsPerBlock, MINB>, kFastWarpsPerBlock * 32, smem);
}

template <class C, int MINB, bool NOOP = false>
void launch_one(const TessDesc& T, const WorkList& W, int nblocks, cudaStream_t s) {
  k_clip_sparse<C, kFastWarpsPerBlock, MINB, NOOP>
      <<<nblocks, kFastWarpsPerBlock * 32, sizeof(SparsePoly<C>) * kFastWarpsPerBlock, s>>>(T, W);
}

template <class C, int MINB>
void launch_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess, const WorkList& W, int nblocks,
                    cudaStream_t s) {
  k_clip_sparse_batched<C, kFastWarpsPerBlock, MINB>
      <<<nblocks, kFastWarpsPerBlock * 32, sizeof(SparsePoly<C>) * kFastWarpsPerBlock, s>>>(descs, tess_off,
                                                                                              ntess, W);
}

}  // namespace

cudaError_t clip_sparse_info(bool mixed, int minb, ClipLaunchInfo* info) {
  cudaError_t e = mixed ? setup_one<MixedSparseCount, 6>(nullptr) : setup_one<FastSparseCount, 6>(nullptr);
  if (e != cudaSuccess) return e;
  if (mixed) {
    if (minb == 5) return setup_one<MixedSparse, 5>(info);
    if (minb == 7) return setup_one<MixedSparse, 7>(info);
    return setup_one<MixedSparse, 6>(info);
  }
  // (the walk's variant with batched plane tests has the same launch shape)
  if (minb == 5) {
    e = setup_one<FastSparse, 5, true>(nullptr);
    return e != cudaSuccess ? e : setup_one<FastSparse, 5>(info);
  }
  if (minb == 7) {
    e = setup_one<FastSparse, 7, true>(nullptr);
    return e != cudaSuccess ? e : setup_one<FastSparse, 7>(info);
  }
  e = setup_one<FastSparse, 6, true>(nullptr);
  return e != cudaSuccess ? e : setup_one<FastSparse, 6>(info);
}

// count: the instrumented variant (always at 6 blocks per SM); noop: the
// walk's variant with batched plane tests (plain FP64, uninstrumented)
cudaError_t launch_clip_sparse(const TessDesc& T, const WorkList& W, int nblocks, bool count, bool mixed, int minb,
                               bool noop, cudaStream_t s) {
  if (mixed) {
    if (count) launch_one<MixedSparseCount, 6>(T, W, nblocks, s);
    else if (minb == 5) launch_one<MixedSparse, 5>(T, W, nblocks, s);
    else if (minb == 7) launch_one<MixedSparse, 7>(T, W, nblocks, s);
    else launch_one<MixedSparse, 6>(T, W, nblocks, s);
  } else {
    if (count) launch_one<FastSparseCount, 6>(T, W, nblocks, s);
    else if (noop && minb == 5) launch_one<FastSparse, 5, true>(T, W, nblocks, s);
    else if (noop && minb == 7) launch_one<FastSparse, 7, true>(T, W, nblocks, s);
    else if (noop) launch_one<FastSparse, 6, true>(T, W, nblocks, s);
    else if (minb == 5) launch_one<FastSparse, 5>(T, W, nblocks, s);
    else if (minb == 7) launch_one<FastSparse, 7>(T, W, nblocks, s);
    else launch_one<FastSparse, 6>(T, W, nblocks, s);
  }
  return cudaGetLastError();
}

cudaError_t clip_sparse_batched_setup(bool mixed, int* blocks_per_sm) {
  cudaError_t e = mixed ? setup_batched<MixedSparseCount, kSparseBatchMinBlocks>(nullptr)
                        : setup_batched<FastSparseCount, kSparseBatchMinBlocks>(nullptr);
  if (e != cudaSuccess) return e;
  return mixed ? setup_batched<MixedSparse, kSparseBatchMinBlocks>(blocks_per_sm)
               : setup_batched<FastSparse, kSparseBatchMinBlocks>(blocks_per_sm);
}

cudaError_t launch_clip_sparse_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess, const WorkList& W,
                                       int nblocks, bool count, bool mixed, cudaStream_t s) {
  if (mixed) {
    if (count) launch_batched<MixedSparseCount, kSparseBatchMinBlocks>(descs, tess_off, ntess, W, nblocks, s);
    else launch_batched<MixedSparse, kSparseBatchMinBlocks>(descs, tess_off, ntess, W, nblocks, s);
  } else {
    if (count) launch_batched<FastSparseCount, kSparseBatchMinBlocks>(descs, tess_off, ntess, W, nblocks, s);
    else launch_batched<FastSparse, kSparseBatchMinBlocks>(descs, tess_off, ntess, W, nblocks, s);
  }
  return cudaGetLastError();
}

}  // namespace vd
