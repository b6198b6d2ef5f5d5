// vd_export.cu -- the polytopes of many cells at once: Tessellation::cells and
// Tessellation::map (tessellation.rs:391-412, 524-526) read every cell's
// Cell3DFaces (vertices, face_counts, face_indices, face_neighbors,
// cell_3d_faces.rs:24-34); this pass rebuilds the cells of a range and writes
// them as one CSR per array (export_worker, vd_export.cuh).  Cells beyond the
// shared-memory capacities are rebuilt by the medium configuration, then by
// the large one in global memory, as calculate's tiers do.
//
// Compiled with -fmad=false like the clip kernels: each cell is rebuilt by the
// same compute_cell, so every vertex equals calculate()'s bit for bit.  The
// production clip kernels are separate instantiations and do not change.
#include "vd_export.cuh"

namespace vd {

namespace {

struct NoExtra {
  template <class C>
  __device__ int operator()(const TessDesc&, uint32_t, WarpPoly<C>&, PolyState&) const {
    return kCellOk;
  }
};

template <class C, int PASS>
__global__ void __launch_bounds__(kExportWarps * 32) k_export_cells(const TessDesc T, const ExportArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  export_worker<C, PASS>(T, A, reinterpret_cast<WarpPoly<C>*>(smem)[threadIdx.x >> 5], NoExtra{});
}

// the large-capacity tier: each warp's polytope in a slice of global scratch
template <class C, int PASS>
__global__ void __launch_bounds__(kExportWarps * 32)
    k_export_cells_global(const TessDesc T, const ExportArgs A, WarpPoly<C>* scratch) {
  const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  export_worker<C, PASS>(T, A, scratch[gw], NoExtra{});
}

template <class C, int PASS>
cudaError_t launch_smem(const TessDesc& T, const ExportArgs& A, int num_sms, cudaStream_t s) {
  const size_t smem = sizeof(WarpPoly<C>) * kExportWarps;
  int nblocks = 1;
  cudaError_t e = export_launch_shape(k_export_cells<C, PASS>, smem, A.nitems, num_sms, &nblocks);
  if (e != cudaSuccess) return e;
  k_export_cells<C, PASS><<<nblocks, kExportWarps * 32, smem, s>>>(T, A);
  return cudaGetLastError();
}

template <int PASS>
cudaError_t launch_tier(const TessDesc& T, const ExportArgs& A, int tier, int num_sms, void* scratch, int nwarps,
                        cudaStream_t s) {
  if (tier == 0) return launch_smem<FastCfg, PASS>(T, A, num_sms, s);
  if (tier == 1) return launch_smem<MedCfgNC, PASS>(T, A, num_sms, s);
  k_export_cells_global<BigCfg, PASS><<<nwarps / kExportWarps, kExportWarps * 32, 0, s>>>(
      T, A, reinterpret_cast<WarpPoly<BigCfg>*>(scratch));
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_export_cells(const TessDesc& T, const ExportArgs& A, int pass, int tier, int num_sms,
                                void* scratch, int nwarps, cudaStream_t s) {
  return pass == 0 ? launch_tier<0>(T, A, tier, num_sms, scratch, nwarps, s)
                   : launch_tier<1>(T, A, tier, num_sms, scratch, nwarps, s);
}

}  // namespace vd
