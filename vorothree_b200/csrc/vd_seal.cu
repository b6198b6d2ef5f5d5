// vd_seal.cu -- the second passes of Tessellation::calculate_sealed and
// Tessellation::prune_boundaries (tessellation.rs:234-385).
//
// Both work on the cells that have a face on a curved wall.  A warp rebuilds
// such a cell with compute_cell (the same polytope calculate built), then
//  - seal: for every face neighbour j (face order, repeats kept) and every
//    curved wall both cells touch (wall order), asks the wall for its tangent
//    plane at j's generator and clips the cell with it when the cell's own
//    generator lies on the plane's valid side; then finalizes the cell;
//  - prune: re-applies those seal clips when the cells are sealed, then for
//    every distinct face neighbour j and every curved wall both cells touch,
//    logs the vertices shared by the cell's faces on the wall and its faces
//    towards j (Cell::shared_vertices, cell_3d_faces.rs:536-565).
// The topology the seal pass reads is a snapshot of calculate's result taken
// before any cell changes, as the reference collects it first.
//
// These kernels are separate instantiations: the production clip kernel's
// code is unchanged.  Compiled with -fmad=false, like every FP64 path.
#include "vd_clip.cuh"
#include "vd_clip_block.cuh"
#include "vd_export.cuh"
#include "vd_internal.h"

namespace vd {
namespace {

__device__ __forceinline__ const int32_t* face_list(const int32_t* nf, const int32_t* fnb, const long long* pool_off,
                                                    const int32_t* pool_fnb, int fout, uint32_t i, int* n) {
  *n = nf[i];
  if (*n <= fout) return fnb + (size_t)i * fout;
  if (pool_off[i] < 0) {  // no pool slots (the host reports pool overflow as an error)
    *n = 0;
    return fnb + (size_t)i * fout;
  }
  return pool_fnb + pool_off[i];
}

// the seal clips of cell i (tessellation.rs:263-311); *nlog gets the number
// of clips that changed the cell, each logged when `log`
template <class C>
__device__ int seal_clips(const TessDesc& T, const SealArgs& A, uint32_t i, WarpPoly<C>& P, PolyState& S, bool log,
                          int* nlog) {
  *nlog = 0;
  const uint32_t mi = A.s_mask[i];
  if (mi == 0) return kCellOk;
  const double gx = T.gen[3 * (size_t)i], gy = T.gen[3 * (size_t)i + 1], gz = T.gen[3 * (size_t)i + 2];
  int nfi;
  const int32_t* fl = face_list(A.s_nf, A.s_fnb, A.s_pool_off, A.s_pool_fnb, A.fout, i, &nfi);
  int cnt = 0;
  for (int q = 0; q < nfi; ++q) {
    const int32_t j = fl[q];
    if (j < 0 || (uint32_t)j >= T.ncells) continue;
    const uint32_t both = mi & A.s_mask[j] & A.curved;
    if (!both) continue;
    const double jx = T.gen[3 * (size_t)j], jy = T.gen[3 * (size_t)j + 1], jz = T.gen[3 * (size_t)j + 2];
    for (int k = 0; k < T.nwalls; ++k) {
      if (!((both >> k) & 1u)) continue;
      double p[3], n[3];
      if (!wall_plane(T.walls[k], jx, jy, jz, p, n)) continue;
      double dot = 0.0;
      dot += (gx - p[0]) * n[0];
      dot += (gy - p[1]) * n[1];
      dot += (gz - p[2]) * n[2];
      if (!(dot <= 1e-9)) continue;
      double r2;
      const int r = warp_clip(P, S, p[0], p[1], p[2], n[0], n[1], n[2], T.walls[k].id, false, gx, gy, gz, &r2);
      if (r == kClipOverflow) return kCellOverflow;
      if (r != kClipNoop) {
        if (log && lane_id() == 0) {
          const unsigned at = atomicAdd(&A.rec_cursor[0], 1u);
          if (at < A.rec_cap) A.seal_rec[at] = SealLogRec{(int32_t)i, cnt, j, T.walls[k].id};
        }
        ++cnt;
      }
    }
  }
  *nlog = cnt;
  return kCellOk;
}

// seal_clips by a whole block (the huge tier, vd_clip_block.cuh); thread 0 logs
template <class C, int NW>
__device__ int seal_clips_block(const TessDesc& T, const SealArgs& A, uint32_t i, WarpPoly<C>& P,
                                BlockShared<NW>& B, PolyState& S, bool log, int* nlog) {
  *nlog = 0;
  const uint32_t mi = A.s_mask[i];
  if (mi == 0) return kCellOk;
  const double gx = T.gen[3 * (size_t)i], gy = T.gen[3 * (size_t)i + 1], gz = T.gen[3 * (size_t)i + 2];
  int nfi;
  const int32_t* fl = face_list(A.s_nf, A.s_fnb, A.s_pool_off, A.s_pool_fnb, A.fout, i, &nfi);
  int cnt = 0;
  for (int q = 0; q < nfi; ++q) {
    const int32_t j = fl[q];
    if (j < 0 || (uint32_t)j >= T.ncells) continue;
    const uint32_t both = mi & A.s_mask[j] & A.curved;
    if (!both) continue;
    const double jx = T.gen[3 * (size_t)j], jy = T.gen[3 * (size_t)j + 1], jz = T.gen[3 * (size_t)j + 2];
    for (int k = 0; k < T.nwalls; ++k) {
      if (!((both >> k) & 1u)) continue;
      double p[3], n[3];
      if (!wall_plane(T.walls[k], jx, jy, jz, p, n)) continue;
      double dot = 0.0;
      dot += (gx - p[0]) * n[0];
      dot += (gy - p[1]) * n[1];
      dot += (gz - p[2]) * n[2];
      if (!(dot <= 1e-9)) continue;
      double r2;
      const int r = block_clip<C, NW>(P, B, S, p[0], p[1], p[2], n[0], n[1], n[2], T.walls[k].id, false, gx, gy, gz, &r2);
      if (r == kClipOverflow) return kCellOverflow;
      if (r != kClipNoop) {
        if (log && threadIdx.x == 0) {
          const unsigned at = atomicAdd(&A.rec_cursor[0], 1u);
          if (at < A.rec_cap) A.seal_rec[at] = SealLogRec{(int32_t)i, cnt, j, T.walls[k].id};
        }
        ++cnt;
      }
    }
  }
  *nlog = cnt;
  return kCellOk;
}

// Cell::shared_vertices(a, b) on the warp's polytope, logged as one prune
// entry (lane 0; a diagnostic pass, not a throughput path).  o2n and lidmap
// are free between clips and serve as per-vertex flags and the order list.
template <class C>
__device__ int prune_shared(const SealArgs& A, uint32_t i, int32_t a, int32_t b, int seq, int pseq,
                            WarpPoly<C>& P, const PolyState& S) {
  int m = 0;
  if (lane_id() == 0) {
    const int cb = S.cb;
    for (int v = 0; v < S.nv; ++v) P.o2n[v] = 0;
    int na = 0;
    for (int f = 0; f < S.nf; ++f) {
      const int32_t x = P.fn[cb][f];
      if (x != a && x != b) continue;
      for (int e = P.fs[cb][f]; e < P.fs[cb][f + 1]; ++e) {
        const int v = P.fi[cb][e];
        if (x == a && !(P.o2n[v] & 1)) {
          P.o2n[v] = (typename C::VId)(P.o2n[v] | 1);
          P.lidmap[na++] = (typename C::VId)v;
        }
        if (x == b) P.o2n[v] = (typename C::VId)(P.o2n[v] | 2);
      }
    }
    for (int k = 0; k < na; ++k) {
      const int v = P.lidmap[k];
      if (!(P.o2n[v] & 2)) continue;
      const unsigned at = atomicAdd(&A.rec_cursor[1], 1u);
      if (at < A.pos_cap) A.prune_pos[at] = PrunePos{(int32_t)i, pseq + m, P.vx[v], P.vy[v], P.vz[v]};
      ++m;
    }
    if (m > 0) {
      const unsigned at = atomicAdd(&A.rec_cursor[0], 1u);
      if (at < A.rec_cap) A.prune_rec[at] = PruneRec{(int32_t)i, seq, b, a, m, pseq};
    }
  }
  m = __shfl_sync(kFull, m, 0);
  __syncwarp();
  return m;
}

// prune_boundaries for cell i (tessellation.rs:355-378) on the current cells
template <class C>
__device__ void prune_cell(const TessDesc& T, const SealArgs& A, uint32_t i, WarpPoly<C>& P, const PolyState& S) {
  const uint32_t mi = A.c_mask[i];
  int nfi;
  const int32_t* fl = face_list(A.c_nf, A.c_fnb, A.c_pool_off, A.c_pool_fnb, A.fout, i, &nfi);
  int seq = 0, pseq = 0;
  for (int q = 0; q < nfi; ++q) {
    const int32_t j = fl[q];
    if (j < 0 || (uint32_t)j >= T.ncells) continue;
    bool seen = false;  // neighbours are taken once, at their first face
    for (int q2 = 0; q2 < q && !seen; ++q2) seen = fl[q2] == j;
    if (seen) continue;
    const uint32_t both = mi & A.c_mask[j] & A.curved;
    for (int k = 0; k < T.nwalls; ++k) {
      if (!((both >> k) & 1u)) continue;
      const int m = prune_shared(A, i, T.walls[k].id, j, seq, pseq, P, S);
      if (m > 0) {
        ++seq;
        pseq += m;
      }
    }
  }
  if (lane_id() == 0) {
    A.cnt[i] = seq;
    A.pcnt[i] = pseq;
  }
}

template <class C>
__device__ void seal_worker(const TessDesc& T, const WorkList& W, const SealArgs& A, WarpPoly<C>& P) {
  const unsigned lane = lane_id();
  if constexpr (C::COUNT) {
    if (lane < kNumCounters) P.cnt[lane] = 0;
  }
  __syncwarp();
  while (true) {
    unsigned idx = 0;
    if (lane == 0) idx = atomicAdd(W.cursor, 1u);
    idx = __shfl_sync(kFull, idx, 0);
    if (idx >= W.nitems) break;
    const uint32_t cell = W.items[idx];
    PolyState S;
    int st = compute_cell<C>(T, cell, P, S);
    int nlog = 0;
    if (st == kCellOk && (A.mode == 1 || A.sealed)) st = seal_clips<C>(T, A, cell, P, S, A.mode == 1, &nlog);
    if (st == kCellOk) {
      if (A.mode == 1) {
        finalize_cell<C>(T, cell, P, S);
        if (W.ex_verts) export_cell<C>(W, P, S);
        if (lane == 0 && A.cnt) A.cnt[cell] = nlog;
      } else {
        prune_cell<C>(T, A, cell, P, S);
      }
    } else if (lane == 0) {
      if (st == kCellOverflow && W.ovf_list) W.ovf_list[atomicAdd(W.ovf_count, 1u)] = cell;
      if (st == kCellTable && W.tab_list) W.tab_list[atomicAdd(W.tab_count, 1u)] = cell;
    }
    __syncwarp();
  }
}

// the seal / prune pass's huge tier: a thread block per cell
template <class C, int NW>
__global__ void __launch_bounds__(NW * 32)
    k_seal_block(const TessDesc T, const WorkList W, const SealArgs A, WarpPoly<C>* polys) {
  __shared__ BlockShared<NW> B;
  WarpPoly<C>& P = polys[blockIdx.x];
  const unsigned lane = lane_id();
  const int w = (int)(threadIdx.x >> 5);
  while (true) {
    if (threadIdx.x == 0) B.idx = atomicAdd(W.cursor, 1u);
    __syncthreads();
    const unsigned idx = B.idx;
    __syncthreads();
    if (idx >= W.nitems) break;
    const uint32_t cell = W.items[idx];
    PolyState S;
    int st = compute_cell_block<C, NW>(T, cell, P, B, S);
    int nlog = 0;
    if (st == kCellOk && (A.mode == 1 || A.sealed))
      st = seal_clips_block<C, NW>(T, A, cell, P, B, S, A.mode == 1, &nlog);
    __syncthreads();
    if (w == 0) {
      if (st == kCellOk) {
        if (A.mode == 1) {
          finalize_cell<C>(T, cell, P, S);
          if (W.ex_verts) export_cell<C>(W, P, S);
          if (lane == 0 && A.cnt) A.cnt[cell] = nlog;
        } else {
          prune_cell<C>(T, A, cell, P, S);
        }
      } else if (lane == 0) {
        if (st == kCellOverflow && W.ovf_list) W.ovf_list[atomicAdd(W.ovf_count, 1u)] = cell;
        if (st == kCellTable && W.tab_list) W.tab_list[atomicAdd(W.tab_count, 1u)] = cell;
      }
    }
    __syncthreads();
  }
}

template <class C, int WPB, int MINB>
__global__ void __launch_bounds__(WPB * 32, MINB) k_seal_fast(const TessDesc T, const WorkList W, const SealArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  WarpPoly<C>* polys = reinterpret_cast<WarpPoly<C>*>(smem);
  seal_worker<C>(T, W, A, polys[threadIdx.x >> 5]);
}

template <class C>
__global__ void __launch_bounds__(128) k_seal_big(const TessDesc T, const WorkList W, const SealArgs A,
                                                  WarpPoly<C>* scratch) {
  const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  seal_worker<C>(T, W, A, scratch[gw]);
}

// per cell: bit k set when wall k's id is among the cell's face neighbours
// and the first wall with that id is curved (walls.iter().find,
// tessellation.rs:250-256)
__global__ void k_curved_mask(const int32_t* nf, const int32_t* fnb, const long long* pool_off,
                              const int32_t* pool_fnb, int fout, uint32_t n, const TessDesc T, uint32_t first_curved,
                              uint32_t* mask) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c;
    const int32_t* fl = face_list(nf, fnb, pool_off, pool_fnb, fout, i, &c);
    uint32_t m = 0;
    for (int q = 0; q < c; ++q) {
      const int32_t x = fl[q];
      if (x >= 0) continue;
      for (int k = 0; k < T.nwalls; ++k)
        if (T.walls[k].id == x && ((first_curved >> k) & 1u)) m |= 1u << k;
    }
    mask[i] = m;
  }
}

// places the log records by (cell, seq) after the per-cell counts are scanned
__global__ void k_seal_log_place(const SealLogRec* rec, uint32_t nrec, const long long* off, int32_t* out) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nrec; r += gridDim.x * blockDim.x) {
    const SealLogRec x = rec[r];
    const long long o = 3 * (off[x.cell] + x.seq);
    out[o] = x.cell;
    out[o + 1] = x.nbr;
    out[o + 2] = x.wall;
  }
}

__global__ void k_prune_log_place(const PruneRec* rec, uint32_t nrec, const PrunePos* pos, uint32_t npos,
                                  const long long* off, const long long* poff, int32_t* out, double* out_pos) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nrec; r += gridDim.x * blockDim.x) {
    const PruneRec x = rec[r];
    const long long o = 4 * (off[x.cell] + x.seq);
    out[o] = x.cell;
    out[o + 1] = x.nbr;
    out[o + 2] = x.wall;
    out[o + 3] = x.count;
  }
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < npos; r += gridDim.x * blockDim.x) {
    const PrunePos x = pos[r];
    const long long o = 3 * (poff[x.cell] + x.pseq);
    out_pos[o] = x.x;
    out_pos[o + 1] = x.y;
    out_pos[o + 2] = x.z;
  }
}

constexpr int kSealMinBlocks = 7;

}  // namespace

cudaError_t seal_setup() {
  return cudaFuncSetAttribute(k_seal_fast<FastCfg, kFastWarpsPerBlock, kSealMinBlocks>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(sizeof(WarpPoly<FastCfg>) * kFastWarpsPerBlock));
}

cudaError_t launch_seal_fast(const TessDesc& T, const WorkList& W, const SealArgs& A, int nblocks, cudaStream_t s) {
  const size_t smem = sizeof(WarpPoly<FastCfg>) * kFastWarpsPerBlock;
  k_seal_fast<FastCfg, kFastWarpsPerBlock, kSealMinBlocks><<<nblocks, kFastWarpsPerBlock * 32, smem, s>>>(T, W, A);
  return cudaGetLastError();
}

cudaError_t launch_seal_big(const TessDesc& T, const WorkList& W, const SealArgs& A, void* scratch, int nwarps,
                            cudaStream_t s) {
  k_seal_big<BigCfg><<<nwarps / 4, 128, 0, s>>>(T, W, A, reinterpret_cast<WarpPoly<BigCfg>*>(scratch));
  return cudaGetLastError();
}

cudaError_t launch_seal_block(const TessDesc& T, const WorkList& W, const SealArgs& A, void* scratch, int nblocks,
                              cudaStream_t s) {
  WarpPoly<HugeCfg>* polys = reinterpret_cast<WarpPoly<HugeCfg>*>(scratch);
  k_seal_block<HugeCfg, kHugeBlockWarps><<<nblocks, kHugeBlockWarps * 32, 0, s>>>(T, W, A, polys);
  return cudaGetLastError();
}

cudaError_t launch_curved_mask(const int32_t* nf, const int32_t* fnb, const long long* pool_off,
                               const int32_t* pool_fnb, int fout, uint32_t n, const TessDesc& T,
                               uint32_t first_curved, uint32_t* mask, int nblocks, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_curved_mask<<<nblocks, 256, 0, s>>>(nf, fnb, pool_off, pool_fnb, fout, n, T, first_curved, mask);
  return cudaGetLastError();
}

cudaError_t launch_seal_log_place(const SealLogRec* rec, uint32_t nrec, const long long* off, int32_t* out,
                                  int nblocks, cudaStream_t s) {
  if (nrec == 0) return cudaSuccess;
  k_seal_log_place<<<nblocks, 256, 0, s>>>(rec, nrec, off, out);
  return cudaGetLastError();
}

cudaError_t launch_prune_log_place(const PruneRec* rec, uint32_t nrec, const PrunePos* pos, uint32_t npos,
                                   const long long* off, const long long* poff, int32_t* out, double* out_pos,
                                   int nblocks, cudaStream_t s) {
  if (nrec == 0 && npos == 0) return cudaSuccess;
  k_prune_log_place<<<nblocks, 256, 0, s>>>(rec, nrec, pos, npos, off, poff, out, out_pos);
  return cudaGetLastError();
}

// bulk export of a sealed tessellation: every cell rebuilt with its seal
// clips (none for a cell without a curved-wall face), nothing logged
namespace {

struct SealExtra {
  SealArgs A;
  template <class C>
  __device__ int operator()(const TessDesc& T, uint32_t cell, WarpPoly<C>& P, PolyState& S) const {
    int nlog = 0;
    return seal_clips<C>(T, A, cell, P, S, false, &nlog);
  }
};

template <class C, int PASS>
__global__ void __launch_bounds__(kExportWarps * 32)
    k_seal_export(const TessDesc T, const ExportArgs E, const SealArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  export_worker<C, PASS>(T, E, reinterpret_cast<WarpPoly<C>*>(smem)[threadIdx.x >> 5], SealExtra{A});
}

template <class C, int PASS>
__global__ void __launch_bounds__(kExportWarps * 32)
    k_seal_export_global(const TessDesc T, const ExportArgs E, const SealArgs A, WarpPoly<C>* scratch) {
  const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  export_worker<C, PASS>(T, E, scratch[gw], SealExtra{A});
}

template <class C, int PASS>
cudaError_t seal_export_smem(const TessDesc& T, const ExportArgs& E, const SealArgs& A, int num_sms,
                             cudaStream_t s) {
  const size_t smem = sizeof(WarpPoly<C>) * kExportWarps;
  int nblocks = 1;
  cudaError_t e = export_launch_shape(k_seal_export<C, PASS>, smem, E.nitems, num_sms, &nblocks);
  if (e != cudaSuccess) return e;
  k_seal_export<C, PASS><<<nblocks, kExportWarps * 32, smem, s>>>(T, E, A);
  return cudaGetLastError();
}

template <int PASS>
cudaError_t seal_export_pass(const TessDesc& T, const ExportArgs& E, const SealArgs& A, int tier, int num_sms,
                             void* scratch, int nwarps, cudaStream_t s) {
  if (tier == 0) return seal_export_smem<FastCfg, PASS>(T, E, A, num_sms, s);
  if (tier == 1) return seal_export_smem<MedCfgNC, PASS>(T, E, A, num_sms, s);
  k_seal_export_global<BigCfg, PASS><<<nwarps / kExportWarps, kExportWarps * 32, 0, s>>>(
      T, E, A, reinterpret_cast<WarpPoly<BigCfg>*>(scratch));
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_seal_export_cells(const TessDesc& T, const ExportArgs& E, const SealArgs& A, int pass, int tier,
                                     int num_sms, void* scratch, int nwarps, cudaStream_t s) {
  return pass == 0 ? seal_export_pass<0>(T, E, A, tier, num_sms, scratch, nwarps, s)
                   : seal_export_pass<1>(T, E, A, tier, num_sms, scratch, nwarps, s);
}

}  // namespace vd
