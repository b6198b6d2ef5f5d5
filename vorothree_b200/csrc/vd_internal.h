// vd_internal.h -- interface between the host library and the kernel
// translation units (not part of the public C ABI).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/voronoid_b200.h"
#include "vd_common.cuh"

namespace vd {

// Fast-path geometry, exported so the host can size launches and buffers.
struct ClipLaunchInfo {
  size_t smem_per_warp;
  int warps_per_block;
  int blocks_per_sm;
  size_t big_scratch_per_warp;
};

// FP64 bit-exact path (vd_kernels_fp64.cu, compiled with -fmad=false)
cudaError_t clip_fp64_info(ClipLaunchInfo* info);
// count: the instrumented variant that maintains the algorithmic event counters
cudaError_t launch_clip_fp64_fast(const TessDesc& T, const WorkList& W, int nblocks, bool count,
                                  cudaStream_t s, bool noop = false);
cudaError_t launch_clip_fp64_big(const TessDesc& T, const WorkList& W, void* scratch, int nwarps,
                                 cudaStream_t s, bool noop = false);

// huge tier (global memory, one thread block per cell): cells beyond the
// large capacities
size_t clip_huge_scratch_per_block();
// narrow: 16-warp blocks (small tessellations), else 32
cudaError_t launch_clip_fp64_huge(const TessDesc& T, const WorkList& W, void* scratch, int nblocks, bool narrow,
                                  cudaStream_t s);
cudaError_t launch_clip_fp64_huge_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess,
                                          const WorkList& W, void* scratch, int nblocks, cudaStream_t s);

// medium-capacity tier (FP64, shared memory) for cells that overflow the fast path
cudaError_t clip_med_setup(ClipLaunchInfo* info);
// count: the instrumented variant (event counters kept)
cudaError_t launch_clip_med(const TessDesc& T, const WorkList& W, int nblocks, bool count, cudaStream_t s, bool noop = false);
cudaError_t launch_clip_med_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess,
                                    const WorkList& W, int nblocks, cudaStream_t s);

// batched mode (descriptors in device memory; see clip_worker_batched)
// *blocks_per_sm: resident blocks of the batched fast kernel
cudaError_t clip_fp64_batched_setup(int* blocks_per_sm);
cudaError_t clip_mixed_batched_setup(int* blocks_per_sm);
cudaError_t launch_clip_fp64_fast_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess,
                                          const WorkList& W, int nblocks, bool count, cudaStream_t s);
cudaError_t launch_clip_mixed_fast_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess,
                                           const WorkList& W, int nblocks, bool count, cudaStream_t s);
cudaError_t launch_clip_fp64_big_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess,
                                         const WorkList& W, void* scratch, int nwarps, cudaStream_t s);

// a device wall from a public wall descriptor (axis normalisation, the
// cone's trigonometry on the host); a polyhedron's planes are appended to
// `planes` (6 doubles each) and the wall records their offset.  Returns
// false with a message for a bad descriptor.
bool wall_from_desc(const vd_wall_desc& d, Wall* w, std::vector<double>* planes, std::string* err);

// bulk polytope export (vd_export.cu): per-cell arrays are indexed by
// cell id - begin
struct ExportArgs {
  const uint32_t* items;  // cell ids to rebuild, in bin order
  uint32_t nitems;
  unsigned int* cursor;   // persistent-warp work counter, zeroed before each pass
  size_t begin;
  int32_t* sizes;         // pass 0: nv, nf, nh of each cell (-1: left to the host)
  const long long* voff;  // pass 1: each cell's first vertex, face and face entry
  const long long* foff;
  const long long* hoff;
  double* verts;
  uint32_t* fc;
  uint32_t* fi;
  int32_t* fn;
};
// tier 0: fast (shared memory), 1: medium (shared memory), 2: large (global
// scratch of nwarps polytopes, a multiple of 4)
cudaError_t launch_export_cells(const TessDesc& T, const ExportArgs& A, int pass, int tier, int num_sms,
                                void* scratch, int nwarps, cudaStream_t s);
// the same for a sealed tessellation (vd_seal.cu): the seal clips applied
cudaError_t launch_seal_export_cells(const TessDesc& T, const ExportArgs& E, const SealArgs& A, int pass, int tier,
                                     int num_sms, void* scratch, int nwarps, cudaStream_t s);

// the generator text format of Tessellation::read_generators (vd_text.cpp):
// false with a message when the text is not UTF-8
bool parse_generators(const char* text, size_t len, std::vector<double>* xyz, std::string* err);

// message returned by vd_last_error(NULL) on the calling thread
void set_thread_error(const char* msg);

// true when an injected allocation failure is pending (vd_debug_fail_allocations);
// consumes it
bool injected_alloc_failure();

// the most warps of large-tier scratch and blocks of huge-tier scratch a
// handle may hold (a server slot's bound); the kernels run with fewer
void set_scratch_caps(vd_tess* t, size_t big_warps, size_t huge_blocks);

// Reserve `bytes` in the library's memory pool on the current device (an
// allocation freed at once; the pool keeps freed memory), so that later
// buffer growth is served from the pool without going to the driver.
cudaError_t reserve_pool(size_t bytes, cudaStream_t s);

// second passes of calculate_sealed / prune_boundaries (vd_seal.cu)
cudaError_t seal_setup();
cudaError_t launch_seal_fast(const TessDesc& T, const WorkList& W, const SealArgs& A, int nblocks, cudaStream_t s);
cudaError_t launch_seal_big(const TessDesc& T, const WorkList& W, const SealArgs& A, void* scratch, int nwarps,
                            cudaStream_t s);
// the seal / prune pass's huge tier (a thread block per cell; scratch as
// for launch_clip_fp64_huge)
cudaError_t launch_seal_block(const TessDesc& T, const WorkList& W, const SealArgs& A, void* scratch, int nblocks,
                              cudaStream_t s);
cudaError_t launch_curved_mask(const int32_t* nf, const int32_t* fnb, const long long* pool_off,
                               const int32_t* pool_fnb, int fout, uint32_t n, const TessDesc& T,
                               uint32_t first_curved, uint32_t* mask, int nblocks, cudaStream_t s);
cudaError_t launch_seal_log_place(const SealLogRec* rec, uint32_t nrec, const long long* off, int32_t* out,
                                  int nblocks, cudaStream_t s);
cudaError_t launch_prune_log_place(const PruneRec* rec, uint32_t nrec, const PrunePos* pos, uint32_t npos,
                                   const long long* off, const long long* poff, int32_t* out, double* out_pos,
                                   int nblocks, cudaStream_t s);

// Mixed path (vd_kernels_mixed.cu)
cudaError_t clip_mixed_info(ClipLaunchInfo* info);

// the shared-memory tier on the slot layout (vd_kernels_sparse.cu): a
// modifying clip rewrites only the faces that lose a vertex; cells it cannot
// finish are listed as overflowing, for the medium tier
// minb: the register budget of 6, 7 or 8 blocks of four warps per SM
cudaError_t clip_sparse_info(bool mixed, int minb, ClipLaunchInfo* info);
// noop: the walk's variant with batched plane tests (TessDesc::noop_run)
cudaError_t launch_clip_sparse(const TessDesc& T, const WorkList& W, int nblocks, bool count, bool mixed, int minb,
                               bool noop, cudaStream_t s);
cudaError_t clip_sparse_batched_setup(bool mixed, int* blocks_per_sm);
// device bytes a committed batch holds beyond its members' buffers
size_t batch_scratch_bytes(int num_sms);
cudaError_t launch_clip_sparse_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess, const WorkList& W,
                                       int nblocks, bool count, bool mixed, cudaStream_t s);
cudaError_t launch_clip_mixed_fast(const TessDesc& T, const WorkList& W, int nblocks, bool count,
                                   cudaStream_t s);

}  // namespace vd
