// vd_export.cu -- the polytopes of many cells at once: Tessellation::cells and
// Tessellation::map (tessellation.rs:391-412, 524-526) read every cell's
// Cell3DFaces (vertices, face_counts, face_indices, face_neighbors,
// cell_3d_faces.rs:24-34); this pass rebuilds the cells of a range and writes
// them as one CSR per array (export_worker, vd_export.cuh).
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

template <int PASS>
cudaError_t launch_pass(const TessDesc& T, const ExportArgs& A, int num_sms, cudaStream_t s) {
  const size_t smem = sizeof(WarpPoly<FastCfg>) * kExportWarps;
  int nblocks = 1;
  cudaError_t e = export_launch_shape(k_export_cells<FastCfg, PASS>, smem, A.nitems, num_sms, &nblocks);
  if (e != cudaSuccess) return e;
  k_export_cells<FastCfg, PASS><<<nblocks, kExportWarps * 32, smem, s>>>(T, A);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_export_cells(const TessDesc& T, const ExportArgs& A, int pass, int num_sms, cudaStream_t s) {
  return pass == 0 ? launch_pass<0>(T, A, num_sms, s) : launch_pass<1>(T, A, num_sms, s);
}

}  // namespace vd
