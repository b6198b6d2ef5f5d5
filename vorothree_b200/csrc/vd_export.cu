// vd_export.cu -- the polytopes of many cells at once: Tessellation::cells and
// Tessellation::map (tessellation.rs:391-412, 524-526) read every cell's
// Cell3DFaces (vertices, face_counts, face_indices, face_neighbors,
// cell_3d_faces.rs:24-34); this pass rebuilds the cells of a range and writes
// them as one CSR per array.
//
// Compiled with -fmad=false like the clip kernels: each cell is rebuilt by the
// same compute_cell, so every vertex equals calculate()'s bit for bit.  Pass 0
// writes each cell's sizes; the host turns them into offsets; pass 1 rebuilds
// the cells and writes each polytope at its offsets.  A cell that does not
// finish in the shared-memory capacities is marked (-1) and left to the
// host, which exports it through get_cell's tiers.
#include <algorithm>

#include "vd_clip.cuh"
#include "vd_internal.h"

namespace vd {

namespace {

constexpr int kExportWarps = 4;

template <class C, int PASS>
__global__ void __launch_bounds__(kExportWarps * 32) k_export_cells(const TessDesc T, const ExportArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  WarpPoly<C>& P = reinterpret_cast<WarpPoly<C>*>(smem)[threadIdx.x >> 5];
  const unsigned lane = lane_id();
  while (true) {
    unsigned idx = 0;
    if (lane == 0) idx = atomicAdd(A.cursor, 1u);
    idx = __shfl_sync(kFull, idx, 0);
    if (idx >= A.nitems) break;
    const uint32_t cell = A.items[idx];
    const size_t k = (size_t)cell - A.begin;
    PolyState S;
    const int st = compute_cell<C>(T, cell, P, S);
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

template <int PASS>
cudaError_t launch_pass(const TessDesc& T, const ExportArgs& A, int num_sms, cudaStream_t s) {
  const size_t smem = sizeof(WarpPoly<FastCfg>) * kExportWarps;
  cudaError_t e = cudaFuncSetAttribute(k_export_cells<FastCfg, PASS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_export_cells<FastCfg, PASS>, kExportWarps * 32, smem);
  if (e != cudaSuccess) return e;
  const size_t warps = A.nitems;
  const int nblocks = (int)std::max<size_t>(
      1, std::min<size_t>((warps + kExportWarps - 1) / kExportWarps, (size_t)num_sms * std::max(1, per_sm)));
  k_export_cells<FastCfg, PASS><<<nblocks, kExportWarps * 32, smem, s>>>(T, A);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_export_cells(const TessDesc& T, const ExportArgs& A, int pass, int num_sms, cudaStream_t s) {
  return pass == 0 ? launch_pass<0>(T, A, num_sms, s) : launch_pass<1>(T, A, num_sms, s);
}

}  // namespace vd
