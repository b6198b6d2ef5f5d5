// vd_export.cuh -- one warp's share of a bulk polytope export pass (the
// kernels are in vd_export.cu, and in vd_seal.cu for sealed tessellations).
// Pass 0 writes each cell's sizes (nv, nf, nh; -1 when the cell did not finish
// in the shared-memory capacities, left to the host); pass 1 rebuilds the
// cell and writes its polytope at the offsets the host derived from pass 0.
#pragma once
#include "vd_clip.cuh"
#include "vd_internal.h"

namespace vd {

constexpr int kExportWarps = 4;

// extra(T, cell, P, S) runs after compute_cell on a finished cell (the seal
// clips of a sealed tessellation) and returns the cell's status
template <class C, int PASS, class Extra>
__device__ void export_worker(const TessDesc& T, const ExportArgs& A, WarpPoly<C>& P, const Extra& extra) {
  const unsigned lane = lane_id();
  while (true) {
    unsigned idx = 0;
    if (lane == 0) idx = atomicAdd(A.cursor, 1u);
    idx = __shfl_sync(kFull, idx, 0);
    if (idx >= A.nitems) break;
    const uint32_t cell = A.items[idx];
    const size_t k = (size_t)cell - A.begin;
    PolyState S;
    int st = compute_cell<C>(T, cell, P, S);
    if (st == kCellOk) st = extra(T, cell, P, S);
    if (PASS == 0) {
      if (lane == 0) {
        A.sizes[3 * k] = st == kCellOk ? S.nv : -1;
        A.sizes[3 * k + 1] = st == kCellOk ? S.nf : -1;
        A.sizes[3 * k + 2] = st == kCellOk ? S.nh : -1;
      }
    } else if (st == kCellOk && S.nv == A.voff[k + 1] - A.voff[k] && S.nf == A.foff[k + 1] - A.foff[k] &&
               S.nh == A.hoff[k + 1] - A.hoff[k]) {
      // (the rebuild is deterministic, so the sizes always match pass 0's;
      // the check keeps every write inside the cell's slots regardless)
      double* v = A.verts + 3 * A.voff[k];
      for (int q = lane; q < S.nv; q += 32) {
        v[3 * q] = P.vx[q];
        v[3 * q + 1] = P.vy[q];
        v[3 * q + 2] = P.vz[q];
      }
      uint32_t* fc = A.fc + A.foff[k];
      int32_t* fn = A.fn + A.foff[k];
      for (int f = lane; f < S.nf; f += 32) {
        fc[f] = (uint32_t)(P.fs[S.cb][f + 1] - P.fs[S.cb][f]);
        fn[f] = P.fn[S.cb][f];
      }
      uint32_t* fi = A.fi + A.hoff[k];
      for (int h = lane; h < S.nh; h += 32) fi[h] = P.fi[S.cb][h];
    }
    __syncwarp();
  }
}

// grid for an export kernel: persistent warps, at most what fits at once
template <class K>
cudaError_t export_launch_shape(K kernel, size_t smem, uint32_t nitems, int num_sms, int* nblocks) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kExportWarps * 32, smem);
  if (e != cudaSuccess) return e;
  const size_t want = ((size_t)nitems + kExportWarps - 1) / kExportWarps;
  const size_t cap = (size_t)num_sms * (size_t)(per_sm > 0 ? per_sm : 1);
  *nblocks = (int)(want < 1 ? 1 : (want < cap ? want : cap));
  return cudaSuccess;
}

}  // namespace vd
