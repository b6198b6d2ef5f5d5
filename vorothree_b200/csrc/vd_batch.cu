// vd_batch.cu -- many independent tessellations in one persistent launch.
//
// A vd_batch holds the members' generators, bins, search orders and outputs
// concatenated in HBM, one TessDesc per member in device memory.  Binning,
// the wall filter, the Lloyd update and the clip kernels all run over the
// whole batch at once; the clip kernel's persistent warps pull cells of every
// member from one work counter, so uneven member sizes balance on their own.
// A Lloyd step (relax -> re-filter -> re-bin -> calculate) is a fixed kernel
// sequence whose sizes live in device memory, so it is captured once in a
// CUDA graph and replayed.
//
// Every member computes exactly what a vd_tess with the same bounds, grid,
// walls and generators computes (same kernels, same arithmetic), which the
// batch tests check bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/voronoid_b200.h"
#include "vd_binning.cuh"
#include "vd_clip.cuh"
#include "vd_internal.h"
#include "vd_order.h"

using namespace vd;

namespace vd_batch_impl {

template <typename T>
struct Buf {
  T* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (vd::injected_alloc_failure()) return cudaErrorMemoryAllocation;
    const size_t want = std::max<size_t>(n, 1);
    cudaError_t e = cudaMalloc(&p, want * sizeof(T));
    if (e == cudaSuccess) cap = want;
    else p = nullptr;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

struct Member {
  Grid g;
  std::vector<Wall> walls;
  std::vector<double> pts;
  int k = 8;
  bool complete = false;
  double bound = 0.0;
  std::vector<Offset> order;
};

// device-side bases the descriptor update derives member pointers from
struct Bases {
  double* gen;
  uint32_t* bin_of;
  uint32_t* bin_start;
  double* vol;
  double* cen;
  int32_t* nfaces;
  int32_t* nverts;
  int32_t* fnb;
  double* farea;
  uint8_t* status;
  long long* pool_off;
  int fout;
};

// ---- batched kernels (the single-tessellation ones with a member lookup) ----
__global__ void k_bwall_flags(const double* __restrict__ in, const uint32_t* off, int ntess,
                              const uint32_t* total_dev, uint32_t nmax, const TessDesc* descs,
                              uint32_t* flags) {
  const uint32_t total = *total_dev;
  // flags[nmax] stays 0 so the scan's last entry is the kept total
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g <= nmax; g += gridDim.x * blockDim.x) {
    uint32_t f = 0;
    if (g < total) {
      const TessDesc& T = descs[find_tess(off, ntess, g)];
      const double x = in[3 * (size_t)g], y = in[3 * (size_t)g + 1], z = in[3 * (size_t)g + 2];
      bool ok = true;
      for (int k = 0; k < T.nwalls && ok; ++k) ok = wall_contains(T.walls[k], T.planes, x, y, z);
      f = ok ? 1u : 0u;
    }
    flags[g] = f;
  }
}

// new member offsets from the compaction scan: member t starts at the
// number of rows kept before its old start
__global__ void k_boffsets(const uint32_t* old_off, const uint32_t* pos, int ntess, uint32_t* new_off,
                           uint32_t* total_dev) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= ntess; t += gridDim.x * blockDim.x) {
    const uint32_t o = pos[old_off[t]];
    new_off[t] = o;
    if (t == ntess) *total_dev = o;
  }
}

__global__ void k_bdesc_update(TessDesc* descs, int ntess, const uint32_t* off, const uint32_t* bin_off,
                               const Bases B) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntess; t += gridDim.x * blockDim.x) {
    TessDesc& T = descs[t];
    const size_t o = off[t];
    T.ncells = off[t + 1] - off[t];
    T.gen = B.gen + 3 * o;
    T.bin_of = B.bin_of + o;
    T.bin_start = B.bin_start + bin_off[t];
    T.vol = B.vol + o;
    T.cen = B.cen + 3 * o;
    T.nfaces = B.nfaces + o;
    T.nverts = B.nverts + o;
    T.fnb = B.fnb + o * (size_t)B.fout;
    T.farea = B.farea + o * (size_t)B.fout;
    T.status = B.status + o;
    T.pool_off = B.pool_off + o;
  }
}

__global__ void k_bbin_count(const double* __restrict__ gen, const uint32_t* off, int ntess,
                             const uint32_t* total_dev, const TessDesc* descs, const uint32_t* bin_off,
                             uint32_t* __restrict__ bin_of, uint32_t* counts) {
  const uint32_t total = *total_dev;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    const int t = find_tess(off, ntess, g);
    const uint32_t b = bin_index(descs[t].grid, gen[3 * (size_t)g], gen[3 * (size_t)g + 1], gen[3 * (size_t)g + 2]);
    bin_of[g] = b;
    atomicAdd(&counts[bin_off[t] + b], 1u);
  }
}

__global__ void k_bbin_scatter(const uint32_t* __restrict__ bin_of, const uint32_t* off, int ntess,
                               const uint32_t* total_dev, const uint32_t* bin_off, uint32_t* cursor,
                               uint32_t* __restrict__ ids) {
  const uint32_t total = *total_dev;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    const int t = find_tess(off, ntess, g);
    ids[atomicAdd(&cursor[bin_off[t] + bin_of[g]], 1u)] = g;
  }
}

// bin-ordered copy; ids are member-local (the cell id within its tessellation)
__global__ void k_bgather(const uint32_t* __restrict__ ids, const double* __restrict__ gen, const uint32_t* off,
                          int ntess, const uint32_t* total_dev, SortedGen* __restrict__ out) {
  const uint32_t total = *total_dev;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    const uint32_t g = ids[k];
    const int t = find_tess(off, ntess, g);
    SortedGen s;
    s.x = gen[3 * (size_t)g];
    s.y = gen[3 * (size_t)g + 1];
    s.z = gen[3 * (size_t)g + 2];
    s.id = (long long)(g - off[t]);
    out[k] = s;
  }
}

__global__ void k_brelax(const double* __restrict__ gen, const int32_t* __restrict__ nverts,
                         const double* __restrict__ cen, const uint32_t* total_dev, double* __restrict__ out) {
  const uint32_t total = *total_dev;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const double* src = nverts[i] == 0 ? gen : cen;
    out[3 * (size_t)i] = src[3 * (size_t)i];
    out[3 * (size_t)i + 1] = src[3 * (size_t)i + 1];
    out[3 * (size_t)i + 2] = src[3 * (size_t)i + 2];
  }
}

// control words: work cursors of the three passes, the overflow counts they
// hand on, the search-order list count, and the big-bin sort count
enum : int {
  kBCursor = 0, kBOvf, kBTab, kBBig, kBCursor2, kBMedOvf, kBCursor3, kBBigOvf, kBCursor4, kBHugeOvf, kBCursorF,
  kBFullOvf, kBWords = 12
};
// blocks of the batch's huge tier (one cell each at a time)
constexpr int kBHugeBlocks = 8;

}  // namespace vd_batch_impl

using namespace vd_batch_impl;

struct vd_batch {
  std::string err;
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  int precision = VD_PREC_FP64;
  bool instrument = false;
  std::vector<Member> m;
  std::vector<double> planes;  // plane table of the members' convex-polyhedron walls
  bool committed = false;
  bool calculated = false;

  uint32_t nmax = 0;        // generators at commit (upper bound of every later count)
  uint32_t nbins = 0;       // bins of all members
  std::vector<uint32_t> h_in_off, h_bin_off, h_off;
  ClipLaunchInfo info64{}, infomx{}, infomed{};
  int blocks64 = 0, blocksmx = 0;  // resident blocks per SM of the batched fast kernels
  int blockssp64 = 0, blocksspmx = 0;  // the same on the slot layout
  int fast_layout = VD_FAST_SLOTS;

  Buf<double> d_in, d_gen, d_vol, d_cen, d_farea, d_pool_area;
  Buf<uint32_t> d_flags, d_pos, d_off, d_off_next, d_in_off, d_total, d_bin_off, d_bin_of, d_counts, d_start,
      d_cursor, d_ids, d_ids_tmp, d_big_list, d_list0, d_list1, d_list2, d_list3;
  Buf<SortedGen> d_sorted;
  Buf<Offset> d_order;
  Buf<TessDesc> d_descs;
  Buf<double> d_planes;
  Buf<int32_t> d_nf, d_nv, d_fnb, d_pool_fnb;
  Buf<uint8_t> d_status;
  Buf<long long> d_pool_off;
  Buf<unsigned int> d_ctl, d_tess_flags;
  Buf<unsigned long long> d_counters, d_pool_cursor;
  Buf<unsigned char> d_big, d_huge;
  int big_warps = 0;
  long long pool_cap = 0;
  std::vector<Buf<uint32_t>> scan_pool;

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  unsigned long long counters[kNumCounters] = {};
  unsigned long long table_reruns = 0;
  unsigned long long pool_reruns = 0;  // chains rerun after the face pool grew
};

namespace {

thread_local std::string g_batch_create_error;

int bfail(vd_batch* b, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  else g_batch_create_error = buf;
  return code;
}

#define B_CK(b, call)                                                                             \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return bfail((b), e_ == cudaErrorMemoryAllocation ? VD_ENOMEM : VD_ECUDA, "%s: %s (%s:%d)", \
                   #call, cudaGetErrorString(e_), __FILE__, __LINE__);                             \
  } while (0)

int blocks_for(const vd_batch* b, size_t n, int threads) {
  const size_t want = (n + threads - 1) / threads;
  return (int)std::max<size_t>(1, std::min(want, (size_t)std::max(1, b->num_sms) * 16));
}

int bscan(vd_batch* b, const uint32_t* in, uint32_t* out, size_t n, int level = 0) {
  if (n == 0) return VD_OK;
  const size_t nt = (n + kScanTile - 1) / kScanTile;
  if ((int)b->scan_pool.size() <= level + 1) b->scan_pool.resize(level + 2);
  B_CK(b, b->scan_pool[level].ensure(nt + 1));
  uint32_t* sums = b->scan_pool[level].p;
  k_scan_tiles<uint32_t, uint32_t><<<(unsigned)nt, kScanThreads, 0, b->stream>>>(in, out, n, sums);
  B_CK(b, cudaGetLastError());
  if (nt > 1) {
    B_CK(b, b->scan_pool[level + 1].ensure(nt + 1));
    uint32_t* sscan = b->scan_pool[level + 1].p;
    int r = bscan(b, sums, sscan, nt, level + 2);
    if (r != VD_OK) return r;
    k_scan_add<uint32_t><<<(unsigned)nt, kScanThreads, 0, b->stream>>>(out, n, sscan);
    B_CK(b, cudaGetLastError());
  }
  return VD_OK;
}

Bases bases(vd_batch* b) {
  Bases B;
  B.gen = b->d_gen.p;
  B.bin_of = b->d_bin_of.p;
  B.bin_start = b->d_start.p;
  B.vol = b->d_vol.p;
  B.cen = b->d_cen.p;
  B.nfaces = b->d_nf.p;
  B.nverts = b->d_nv.p;
  B.fnb = b->d_fnb.p;
  B.farea = b->d_farea.p;
  B.status = b->d_status.p;
  B.pool_off = b->d_pool_off.p;
  B.fout = 48;
  return B;
}

// static descriptor parts (grid, walls, search order); the per-step parts are
// written on the device by k_bdesc_update
int upload_static(vd_batch* b) {
  const int nt = (int)b->m.size();
  size_t total_order = 0;
  std::vector<size_t> order_off(nt + 1, 0);
  for (int t = 0; t < nt; ++t) {
    order_off[t] = total_order;
    total_order += b->m[t].order.size();
  }
  order_off[nt] = total_order;
  B_CK(b, b->d_order.ensure(total_order));
  std::vector<Offset> cat(total_order);
  for (int t = 0; t < nt; ++t)
    std::copy(b->m[t].order.begin(), b->m[t].order.end(), cat.begin() + order_off[t]);
  B_CK(b, cudaMemcpyAsync(b->d_order.p, cat.data(), total_order * sizeof(Offset), cudaMemcpyHostToDevice, b->stream));
  B_CK(b, b->d_planes.ensure(std::max<size_t>(b->planes.size(), 1)));
  if (!b->planes.empty())
    B_CK(b, cudaMemcpyAsync(b->d_planes.p, b->planes.data(), b->planes.size() * sizeof(double),
                            cudaMemcpyHostToDevice, b->stream));
  std::vector<TessDesc> d(nt);
  for (int t = 0; t < nt; ++t) {
    TessDesc& T = d[t];
    memset(&T, 0, sizeof(T));
    const Member& M = b->m[t];
    T.grid = M.g;
    T.nwalls = (int)M.walls.size();
    for (int k = 0; k < T.nwalls; ++k) T.walls[k] = M.walls[k];
    T.planes = b->d_planes.p;
    T.order = b->d_order.p + order_off[t];
    T.norder = (int)M.order.size();
    T.order_complete = M.complete ? 1 : 0;
    T.order_bound = M.bound;
    T.sorted = b->d_sorted.p;
    T.fout = 48;
    T.pool_fnb = b->d_pool_fnb.p;
    T.pool_farea = b->d_pool_area.p;
    T.pool_cursor = b->d_pool_cursor.p;
    T.pool_cap = b->pool_cap;
  }
  B_CK(b, cudaMemcpyAsync(b->d_descs.p, d.data(), nt * sizeof(TessDesc), cudaMemcpyHostToDevice, b->stream));
  B_CK(b, cudaStreamSynchronize(b->stream));
  return VD_OK;
}

// wall filter of d_src (laid out by src_off) into d_gen, new offsets into
// d_off, descriptors and bins rebuilt -- all on the stream, sizes on device
int filter_and_bin(vd_batch* b, const double* d_src, const uint32_t* src_off) {
  cudaStream_t s = b->stream;
  const int nt = (int)b->m.size();
  const uint32_t nmax = b->nmax;
  k_bwall_flags<<<blocks_for(b, nmax, 256), 256, 0, s>>>(d_src, src_off, nt, b->d_total.p, nmax, b->d_descs.p,
                                                        b->d_flags.p);
  B_CK(b, cudaGetLastError());
  int r = bscan(b, b->d_flags.p, b->d_pos.p, (size_t)nmax + 1);
  if (r != VD_OK) return r;
  k_compact3<<<blocks_for(b, nmax, 256), 256, 0, s>>>(d_src, nmax, b->d_flags.p, b->d_pos.p, b->d_gen.p);
  B_CK(b, cudaGetLastError());
  k_boffsets<<<blocks_for(b, nt + 1, 256), 256, 0, s>>>(src_off, b->d_pos.p, nt, b->d_off_next.p, b->d_total.p);
  B_CK(b, cudaGetLastError());
  B_CK(b, cudaMemcpyAsync(b->d_off.p, b->d_off_next.p, (nt + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  k_bdesc_update<<<blocks_for(b, nt, 128), 128, 0, s>>>(b->d_descs.p, nt, b->d_off.p, b->d_bin_off.p, bases(b));
  B_CK(b, cudaGetLastError());
  // Algorithm3DGrid::set_generators for every member
  B_CK(b, cudaMemsetAsync(b->d_counts.p, 0, ((size_t)b->nbins + 1) * sizeof(uint32_t), s));
  B_CK(b, cudaMemsetAsync(b->d_ctl.p + kBBig, 0, sizeof(unsigned int), s));
  k_bbin_count<<<blocks_for(b, nmax, 256), 256, 0, s>>>(b->d_gen.p, b->d_off.p, nt, b->d_total.p, b->d_descs.p,
                                                       b->d_bin_off.p, b->d_bin_of.p, b->d_counts.p);
  B_CK(b, cudaGetLastError());
  r = bscan(b, b->d_counts.p, b->d_start.p, (size_t)b->nbins + 1);
  if (r != VD_OK) return r;
  B_CK(b, cudaMemcpyAsync(b->d_cursor.p, b->d_start.p, (size_t)b->nbins * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  k_bbin_scatter<<<blocks_for(b, nmax, 256), 256, 0, s>>>(b->d_bin_of.p, b->d_off.p, nt, b->d_total.p,
                                                         b->d_bin_off.p, b->d_cursor.p, b->d_ids.p);
  B_CK(b, cudaGetLastError());
  k_bin_fix<<<blocks_for(b, b->nbins, 256), 256, 0, s>>>(b->d_start.p, b->nbins, b->d_ids.p, b->d_big_list.p,
                                                        b->d_ctl.p + kBBig);
  B_CK(b, cudaGetLastError());
  k_bin_sort_big<<<std::max(1, b->num_sms), kBigSortThreads, 0, s>>>(b->d_start.p, b->d_big_list.p,
                                                                    b->d_ctl.p + kBBig, b->d_ids.p, b->d_ids_tmp.p);
  B_CK(b, cudaGetLastError());
  k_bgather<<<blocks_for(b, nmax, 256), 256, 0, s>>>(b->d_ids.p, b->d_gen.p, b->d_off.p, nt, b->d_total.p,
                                                    b->d_sorted.p);
  B_CK(b, cudaGetLastError());
  return VD_OK;
}

// The clip chain over a work list: the fast pass, then the medium-capacity
// pass over its overflow list, then the large-capacity pass over what still
// overflows -- every count lives on the device, so the chain can be captured.
// items == nullptr: every cell (the count is the batch total).
int clip_chain(vd_batch* b, const uint32_t* items, uint32_t nitems) {
  cudaStream_t s = b->stream;
  const int nt = (int)b->m.size();
  B_CK(b, cudaMemsetAsync(b->d_ctl.p, 0, 3 * sizeof(unsigned int), s));
  B_CK(b, cudaMemsetAsync(b->d_ctl.p + kBCursor2, 0, 8 * sizeof(unsigned int), s));
  WorkList W;
  memset(&W, 0, sizeof(W));
  W.items = items;
  W.nitems = nitems;
  W.nitems_dev = items ? nullptr : b->d_total.p;
  W.cursor = b->d_ctl.p + kBCursor;
  W.ovf_list = b->d_list0.p;
  W.ovf_count = b->d_ctl.p + kBOvf;
  W.tab_list = b->d_list1.p;
  W.tab_count = b->d_ctl.p + kBTab;
  W.counters = b->d_counters.p;
  W.tess_flags = b->d_tess_flags.p;
  const bool mixed = b->precision == VD_PREC_MIXED;
  if (b->fast_layout == VD_FAST_SLOTS) {
    const int nblocks = std::max(1, b->num_sms * std::max(1, mixed ? b->blocksspmx : b->blockssp64));
    B_CK(b, launch_clip_sparse_batched(b->d_descs.p, b->d_off.p, nt, W, nblocks, b->instrument, mixed, s));
  } else {
    const int nblocks = std::max(1, b->num_sms * std::max(1, mixed ? b->blocksmx : b->blocks64));
    B_CK(b, mixed ? launch_clip_mixed_fast_batched(b->d_descs.p, b->d_off.p, nt, W, nblocks, b->instrument, s)
                  : launch_clip_fp64_fast_batched(b->d_descs.p, b->d_off.p, nt, W, nblocks, b->instrument, s));
  }
  // the slot layout's hand-offs: the full-rewrite first tier (48 faces)
  const uint32_t* med_in = b->d_list0.p;
  unsigned int* med_n = b->d_ctl.p + kBOvf;
  if (b->fast_layout == VD_FAST_SLOTS) {
    WorkList WF = W;
    WF.items = b->d_list0.p;
    WF.nitems = 0;
    WF.nitems_dev = b->d_ctl.p + kBOvf;
    WF.cursor = b->d_ctl.p + kBCursorF;
    WF.ovf_list = b->d_list3.p;
    WF.ovf_count = b->d_ctl.p + kBFullOvf;
    const int nbf = std::max(1, b->num_sms * std::max(1, mixed ? b->blocksmx : b->blocks64));
    B_CK(b, mixed ? launch_clip_mixed_fast_batched(b->d_descs.p, b->d_off.p, nt, WF, nbf, b->instrument, s)
                  : launch_clip_fp64_fast_batched(b->d_descs.p, b->d_off.p, nt, WF, nbf, b->instrument, s));
    med_in = b->d_list3.p;
    med_n = b->d_ctl.p + kBFullOvf;
  }
  // medium capacity (FP64; the same decisions as both precisions)
  WorkList W2 = W;
  W2.items = med_in;
  W2.nitems = 0;
  W2.nitems_dev = med_n;
  W2.cursor = b->d_ctl.p + kBCursor2;
  W2.ovf_list = b->d_list2.p;
  W2.ovf_count = b->d_ctl.p + kBMedOvf;
  B_CK(b, launch_clip_med_batched(b->d_descs.p, b->d_off.p, nt, W2,
                                  std::max(1, b->num_sms * std::max(1, b->infomed.blocks_per_sm)), s));
  // large capacity (global-memory storage)
  WorkList W3 = W;
  W3.items = b->d_list2.p;
  W3.nitems = 0;
  W3.nitems_dev = b->d_ctl.p + kBMedOvf;
  W3.cursor = b->d_ctl.p + kBCursor3;
  W3.ovf_list = b->d_list0.p;
  W3.ovf_count = b->d_ctl.p + kBBigOvf;
  B_CK(b, launch_clip_fp64_big_batched(b->d_descs.p, b->d_off.p, nt, W3, b->d_big.p, b->big_warps, s));
  // huge capacity (a thread block per cell); what overflows here is an error
  WorkList W4 = W;
  W4.items = b->d_list0.p;
  W4.nitems = 0;
  W4.nitems_dev = b->d_ctl.p + kBBigOvf;
  W4.cursor = b->d_ctl.p + kBCursor4;
  W4.ovf_list = b->d_list2.p;
  W4.ovf_count = b->d_ctl.p + kBHugeOvf;
  B_CK(b, launch_clip_fp64_huge_batched(b->d_descs.p, b->d_off.p, nt, W4, b->d_huge.p, kBHugeBlocks, s));
  return VD_OK;
}

int clip_all(vd_batch* b) {
  B_CK(b, cudaMemsetAsync(b->d_pool_cursor.p, 0, sizeof(unsigned long long), b->stream));
  return clip_chain(b, nullptr, 0);
}

void drop_graph(vd_batch* b) {
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->graph_exec = nullptr;
  b->graph = nullptr;
}

// The face pool (face slots of cells with more than 48 faces) was too small
// for the last clip chain: cells that found no room have no face slots and a
// face count of -1.  Grow the pool to what the chain asked for and run the
// whole chain again on the same generators (a captured Lloyd step holds the
// old pool in its descriptors, so it is dropped and captured again later).
int grow_pool_and_rerun(vd_batch* b, unsigned long long used) {
  cudaStream_t s = b->stream;
  const int nt = (int)b->m.size();
  b->pool_cap = std::max<long long>(2 * b->pool_cap, (long long)(used + used / 4));
  B_CK(b, cudaStreamSynchronize(s));
  B_CK(b, b->d_pool_fnb.ensure(b->pool_cap));
  B_CK(b, b->d_pool_area.ensure(b->pool_cap));
  drop_graph(b);
  int r = upload_static(b);
  if (r != VD_OK) return r;
  k_bdesc_update<<<blocks_for(b, nt, 128), 128, 0, s>>>(b->d_descs.p, nt, b->d_off.p, b->d_bin_off.p, bases(b));
  B_CK(b, cudaGetLastError());
  B_CK(b, cudaMemsetAsync(b->d_tess_flags.p, 0, nt * sizeof(unsigned int), s));
  B_CK(b, cudaMemsetAsync(b->d_counters.p, 0, kNumCounters * sizeof(unsigned long long), s));
  ++b->pool_reruns;
  return clip_all(b);
}

// cells that ran off a truncated search order: lengthen that member's table
// and run them again (host loop; rare for uniform inputs); a face pool that
// was too small is grown and the chain rerun
int resolve_tables(vd_batch* b) {
  cudaStream_t s = b->stream;
  const int nt = (int)b->m.size();
  for (int guard = 0; guard < 32; ++guard) {
    unsigned int h[kBWords];
    unsigned long long used = 0;
    B_CK(b, cudaMemcpyAsync(h, b->d_ctl.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    B_CK(b, cudaMemcpyAsync(&used, b->d_pool_cursor.p, sizeof(used), cudaMemcpyDeviceToHost, s));
    B_CK(b, cudaStreamSynchronize(s));
    if (h[kBHugeOvf] > 0) return bfail(b, VD_EOVERFLOW, "%u cells exceed the huge polytope capacity", h[kBHugeOvf]);
    if ((long long)used > b->pool_cap) {
      int r = grow_pool_and_rerun(b, used);
      if (r != VD_OK) return r;
      continue;
    }
    const unsigned ntab = h[kBTab];
    if (ntab == 0) return VD_OK;
    std::vector<unsigned int> flags(nt);
    B_CK(b, cudaMemcpyAsync(flags.data(), b->d_tess_flags.p, nt * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    B_CK(b, cudaStreamSynchronize(s));
    for (int t = 0; t < nt; ++t)
      if (flags[t]) {
        Member& M = b->m[t];
        if (M.complete) return bfail(b, VD_ECUDA, "search order exhausted on a complete table");
        M.k *= 2;
        build_order(M.g, M.k, M.order, M.complete, M.bound);
      }
    B_CK(b, cudaMemsetAsync(b->d_tess_flags.p, 0, nt * sizeof(unsigned int), s));
    int r = upload_static(b);
    if (r != VD_OK) return r;
    // upload_static rewrote whole descriptors: restore the per-step parts
    k_bdesc_update<<<blocks_for(b, nt, 128), 128, 0, s>>>(b->d_descs.p, nt, b->d_off.p, b->d_bin_off.p, bases(b));
    B_CK(b, cudaGetLastError());
    // rerun the listed cells (from a copy: the chain refills the lists)
    B_CK(b, b->d_list3.ensure(b->nmax));
    B_CK(b, cudaMemcpyAsync(b->d_list3.p, b->d_list1.p, ntab * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    r = clip_chain(b, b->d_list3.p, ntab);
    if (r != VD_OK) return r;
    b->table_reruns += ntab;
  }
  return bfail(b, VD_ECUDA, "search-order extension did not converge");
}

int read_offsets(vd_batch* b) {
  const int nt = (int)b->m.size();
  b->h_off.resize(nt + 1);
  B_CK(b, cudaMemcpyAsync(b->h_off.data(), b->d_off.p, (nt + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream));
  B_CK(b, cudaMemcpyAsync(b->counters, b->d_counters.p, sizeof(b->counters), cudaMemcpyDeviceToHost, b->stream));
  B_CK(b, cudaStreamSynchronize(b->stream));
  return VD_OK;
}

// one Lloyd step: Tessellation::relax (tessellation.rs:482-495) then calculate
int lloyd_step(vd_batch* b) {
  k_brelax<<<blocks_for(b, b->nmax, 256), 256, 0, b->stream>>>(b->d_gen.p, b->d_nv.p, b->d_cen.p, b->d_total.p,
                                                              b->d_in.p);
  B_CK(b, cudaGetLastError());
  // the relaxed rows keep the current layout: filter them by the current offsets
  B_CK(b, cudaMemcpyAsync(b->d_in_off.p, b->d_off.p, (b->m.size() + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                          b->stream));
  int r = filter_and_bin(b, b->d_in.p, b->d_in_off.p);
  if (r != VD_OK) return r;
  return clip_all(b);
}

}  // namespace

namespace vd {
// device bytes a committed batch holds beyond its members' own buffers: the
// large tier's warps, the huge tier's blocks and the first face pool
size_t batch_scratch_bytes(int num_sms) {
  ClipLaunchInfo info{};
  clip_fp64_info(&info);
  return (size_t)std::max(4, num_sms * 4) * info.big_scratch_per_warp +
         (size_t)kBHugeBlocks * clip_huge_scratch_per_block() + ((size_t)1 << 20) * 12;
}
}  // namespace vd

extern "C" {

const char* vd_batch_last_error(const vd_batch* b) { return b ? b->err.c_str() : g_batch_create_error.c_str(); }

int vd_batch_create(vd_batch** out) {
  if (!out) return bfail(nullptr, VD_EINVAL, "null argument");
  *out = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return bfail(nullptr, VD_ECUDA, "no CUDA device: %s", cudaGetErrorString(e));
  vd_batch* b = new vd_batch();
  b->device = dev;
  cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = clip_fp64_info(&b->info64);
  if (e == cudaSuccess) e = clip_mixed_info(&b->infomx);
  if (e == cudaSuccess) e = clip_med_setup(&b->infomed);
  if (e == cudaSuccess) e = clip_fp64_batched_setup(&b->blocks64);
  if (e == cudaSuccess) e = clip_mixed_batched_setup(&b->blocksmx);
  if (e == cudaSuccess) e = clip_sparse_batched_setup(false, &b->blockssp64);
  if (e == cudaSuccess) e = clip_sparse_batched_setup(true, &b->blocksspmx);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
  if (e != cudaSuccess) {
    const std::string msg = cudaGetErrorString(e);
    vd_batch_destroy(b);
    return bfail(nullptr, VD_ECUDA, "batch setup: %s", msg.c_str());
  }
  *out = b;
  return VD_OK;
}

int vd_batch_destroy(vd_batch* b) {
  if (!b) return VD_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->d_in.release(); b->d_gen.release(); b->d_vol.release(); b->d_cen.release(); b->d_farea.release();
  b->d_pool_area.release(); b->d_flags.release(); b->d_pos.release(); b->d_off.release(); b->d_off_next.release();
  b->d_in_off.release(); b->d_total.release(); b->d_bin_off.release(); b->d_bin_of.release(); b->d_counts.release();
  b->d_start.release(); b->d_cursor.release(); b->d_ids.release(); b->d_ids_tmp.release(); b->d_big_list.release();
  b->d_list0.release(); b->d_list1.release(); b->d_list2.release(); b->d_list3.release(); b->d_sorted.release(); b->d_order.release();
  b->d_descs.release(); b->d_planes.release(); b->d_nf.release(); b->d_nv.release(); b->d_fnb.release(); b->d_pool_fnb.release();
  b->d_status.release(); b->d_pool_off.release(); b->d_ctl.release(); b->d_tess_flags.release();
  b->d_counters.release(); b->d_pool_cursor.release(); b->d_big.release(); b->d_huge.release();
  for (auto& p : b->scan_pool) p.release();
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return VD_OK;
}

// the members are dropped and the batch takes new ones; device buffers and
// the stream are kept (they only grow), so a batch reused for batches of
// similar size allocates nothing
int vd_batch_reset(vd_batch* b) {
  if (!b) return VD_EINVAL;
  B_CK(b, cudaSetDevice(b->device));
  B_CK(b, cudaStreamSynchronize(b->stream));
  drop_graph(b);
  b->m.clear();
  b->planes.clear();
  b->committed = false;
  b->calculated = false;
  b->nmax = 0;
  b->nbins = 0;
  b->last_ms = 0.f;
  memset(b->counters, 0, sizeof(b->counters));
  b->table_reruns = 0;
  b->pool_reruns = 0;
  return VD_OK;
}

int vd_batch_add(vd_batch* b, const double bmin[3], const double bmax[3], int nx, int ny, int nz,
                 const vd_wall_desc* walls, int nwalls, const double* xyz, size_t n, int* index) {
  if (!b || !bmin || !bmax || (!xyz && n) || (nwalls > 0 && !walls)) return VD_EINVAL;
  if (b->committed) return bfail(b, VD_ESTATE, "batch already committed");
  if (nx <= 0 || ny <= 0 || nz <= 0) return bfail(b, VD_EINVAL, "grid resolution must be positive");
  if (nwalls < 0 || nwalls > kMaxWalls) return bfail(b, VD_EINVAL, "at most %d walls", kMaxWalls);
  Member M;
  const int nn[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) {
    M.g.bmin[a] = bmin[a];
    M.g.bmax[a] = bmax[a];
    M.g.n[a] = nn[a];
    M.g.scale[a] = (double)nn[a] / (bmax[a] - bmin[a]);
    M.g.limit[a] = (double)nn[a] - 1e-5;
    M.g.cs[a] = 1.0 / M.g.scale[a];
  }
  for (int k = 0; k < nwalls; ++k) {
    Wall w;
    std::string err;
    if (!wall_from_desc(walls[k], &w, &b->planes, &err)) return bfail(b, VD_EINVAL, "wall %d: %s", k, err.c_str());
    M.walls.push_back(w);
  }
  M.pts.assign(xyz, xyz + 3 * n);
  const double full = (2.0 * nx + 1) * (2.0 * ny + 1) * (2.0 * nz + 1);
  M.k = full <= 20000.0 ? std::max(nx, std::max(ny, nz)) : 8;
  build_order(M.g, M.k, M.order, M.complete, M.bound);
  b->m.push_back(std::move(M));
  if (index) *index = (int)b->m.size() - 1;
  return VD_OK;
}

int vd_batch_set_precision(vd_batch* b, int precision) {
  if (!b) return VD_EINVAL;
  if (precision != VD_PREC_FP64 && precision != VD_PREC_MIXED) return bfail(b, VD_EINVAL, "unknown precision");
  b->precision = precision;
  drop_graph(b);  // the captured step uses the previous kernel
  return VD_OK;
}

int vd_batch_set_fast_layout(vd_batch* b, int layout) {
  if (!b) return VD_EINVAL;
  if (layout != VD_FAST_SLOTS && layout != VD_FAST_FULL) return bfail(b, VD_EINVAL, "unknown fast-tier layout");
  b->fast_layout = layout;
  drop_graph(b);  // the captured step uses the previous kernel
  return VD_OK;
}

int vd_batch_set_instrumentation(vd_batch* b, int on) {
  if (!b) return VD_EINVAL;
  b->instrument = on != 0;
  return vd_batch_set_precision(b, b->precision);
}

int vd_batch_commit(vd_batch* b) {
  if (!b) return VD_EINVAL;
  if (b->committed) return bfail(b, VD_ESTATE, "batch already committed");
  if (b->m.empty()) return bfail(b, VD_EINVAL, "empty batch");
  B_CK(b, cudaSetDevice(b->device));
  const int nt = (int)b->m.size();
  size_t n = 0, nb = 0;
  b->h_in_off.assign(nt + 1, 0);
  b->h_bin_off.assign(nt + 1, 0);
  for (int t = 0; t < nt; ++t) {
    b->h_in_off[t] = (uint32_t)n;
    b->h_bin_off[t] = (uint32_t)nb;
    n += b->m[t].pts.size() / 3;
    nb += (size_t)b->m[t].g.n[0] * b->m[t].g.n[1] * b->m[t].g.n[2];
    if (n > 0xF0000000ull || nb > 0xF0000000ull) return bfail(b, VD_EINVAL, "batch too large");
  }
  b->h_in_off[nt] = (uint32_t)n;
  b->h_bin_off[nt] = (uint32_t)nb;
  b->nmax = (uint32_t)n;
  b->nbins = (uint32_t)nb;
  const size_t fout = 48;
  B_CK(b, b->d_in.ensure(3 * n));
  B_CK(b, b->d_gen.ensure(3 * n));
  B_CK(b, b->d_flags.ensure(n + 1));
  B_CK(b, b->d_pos.ensure(n + 1));
  B_CK(b, b->d_off.ensure(nt + 1));
  B_CK(b, b->d_off_next.ensure(nt + 1));
  B_CK(b, b->d_in_off.ensure(nt + 1));
  B_CK(b, b->d_total.ensure(1));
  B_CK(b, b->d_bin_off.ensure(nt + 1));
  B_CK(b, b->d_bin_of.ensure(n));
  B_CK(b, b->d_counts.ensure(nb + 1));
  B_CK(b, b->d_start.ensure(nb + 1));
  B_CK(b, b->d_cursor.ensure(nb + 1));
  B_CK(b, b->d_ids.ensure(n));
  B_CK(b, b->d_ids_tmp.ensure(n));
  B_CK(b, b->d_big_list.ensure(nb));
  B_CK(b, b->d_list0.ensure(n));
  B_CK(b, b->d_list1.ensure(n));
  B_CK(b, b->d_list2.ensure(n));
  B_CK(b, b->d_list3.ensure(n));
  B_CK(b, b->d_sorted.ensure(n));
  B_CK(b, b->d_descs.ensure(nt));
  B_CK(b, b->d_vol.ensure(n));
  B_CK(b, b->d_cen.ensure(3 * n));
  B_CK(b, b->d_nf.ensure(n));
  B_CK(b, b->d_nv.ensure(n));
  B_CK(b, b->d_fnb.ensure(n * fout));
  B_CK(b, b->d_farea.ensure(n * fout));
  B_CK(b, b->d_status.ensure(n));
  B_CK(b, b->d_pool_off.ensure(n));
  B_CK(b, b->d_ctl.ensure(kBWords));
  B_CK(b, b->d_tess_flags.ensure(nt));
  B_CK(b, b->d_counters.ensure(kNumCounters));
  B_CK(b, b->d_pool_cursor.ensure(1));
  b->pool_cap = std::max<long long>(b->pool_cap, 1 << 20);  // (a reused batch keeps a grown pool)
  B_CK(b, b->d_pool_fnb.ensure(b->pool_cap));
  B_CK(b, b->d_pool_area.ensure(b->pool_cap));
  b->big_warps = std::max(4, b->num_sms * 4);
  B_CK(b, b->d_big.ensure((size_t)b->big_warps * b->info64.big_scratch_per_warp));
  B_CK(b, b->d_huge.ensure((size_t)kBHugeBlocks * clip_huge_scratch_per_block()));
  cudaStream_t s = b->stream;
  std::vector<double> cat(3 * n);
  for (int t = 0; t < nt; ++t) std::copy(b->m[t].pts.begin(), b->m[t].pts.end(), cat.begin() + 3 * b->h_in_off[t]);
  B_CK(b, cudaMemcpyAsync(b->d_in.p, cat.data(), cat.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  B_CK(b, cudaMemcpyAsync(b->d_in_off.p, b->h_in_off.data(), (nt + 1) * 4, cudaMemcpyHostToDevice, s));
  B_CK(b, cudaMemcpyAsync(b->d_bin_off.p, b->h_bin_off.data(), (nt + 1) * 4, cudaMemcpyHostToDevice, s));
  B_CK(b, cudaMemcpyAsync(b->d_total.p, &b->nmax, 4, cudaMemcpyHostToDevice, s));
  B_CK(b, cudaMemsetAsync(b->d_tess_flags.p, 0, nt * sizeof(unsigned int), s));
  B_CK(b, cudaMemsetAsync(b->d_counters.p, 0, kNumCounters * sizeof(unsigned long long), s));
  int r = upload_static(b);
  if (r != VD_OK) return r;
  // Tessellation::set_generators for every member: wall filter + binning
  r = filter_and_bin(b, b->d_in.p, b->d_in_off.p);
  if (r != VD_OK) return r;
  B_CK(b, cudaStreamSynchronize(s));
  for (auto& M : b->m) std::vector<double>().swap(M.pts);
  b->committed = true;
  return read_offsets(b);
}

int vd_batch_calculate(vd_batch* b) {
  if (!b) return VD_EINVAL;
  if (!b->committed) return bfail(b, VD_ESTATE, "commit the batch first");
  B_CK(b, cudaSetDevice(b->device));
  B_CK(b, cudaMemsetAsync(b->d_counters.p, 0, kNumCounters * sizeof(unsigned long long), b->stream));
  B_CK(b, cudaEventRecord(b->ev0, b->stream));
  int r = clip_all(b);
  if (r != VD_OK) return r;
  r = resolve_tables(b);
  if (r != VD_OK) return r;
  B_CK(b, cudaEventRecord(b->ev1, b->stream));
  B_CK(b, cudaEventSynchronize(b->ev1));
  cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
  b->calculated = true;
  return read_offsets(b);
}

int vd_batch_lloyd(vd_batch* b, int steps) {
  if (!b || steps < 0) return VD_EINVAL;
  if (!b->calculated) return bfail(b, VD_ESTATE, "calculate the batch before relaxing it");
  B_CK(b, cudaSetDevice(b->device));
  cudaStream_t s = b->stream;
  if (!b->graph_exec && steps > 0) {
    // one eager step sizes every scratch buffer; the graph captures the next
    B_CK(b, cudaMemsetAsync(b->d_counters.p, 0, kNumCounters * sizeof(unsigned long long), s));
    B_CK(b, cudaEventRecord(b->ev0, s));
    int r = lloyd_step(b);
    if (r != VD_OK) return r;
    r = resolve_tables(b);
    if (r != VD_OK) return r;
    --steps;
    B_CK(b, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    r = lloyd_step(b);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (r != VD_OK) {
      if (g) cudaGraphDestroy(g);
      return r;
    }
    B_CK(b, e);
    b->graph = g;
    B_CK(b, cudaGraphInstantiate(&b->graph_exec, g, 0));
  } else {
    B_CK(b, cudaMemsetAsync(b->d_counters.p, 0, kNumCounters * sizeof(unsigned long long), s));
    B_CK(b, cudaEventRecord(b->ev0, s));
  }
  for (int i = 0; i < steps; ++i) {
    if (b->graph_exec) {
      B_CK(b, cudaGraphLaunch(b->graph_exec, s));
    } else {  // dropped by a pool growth: the remaining steps run eagerly
      int r = lloyd_step(b);
      if (r != VD_OK) return r;
    }
    int r = resolve_tables(b);
    if (r != VD_OK) return r;
  }
  B_CK(b, cudaEventRecord(b->ev1, s));
  B_CK(b, cudaEventSynchronize(b->ev1));
  cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
  return read_offsets(b);
}

int vd_batch_count(const vd_batch* b, int* ntess) {
  if (!b || !ntess) return VD_EINVAL;
  *ntess = (int)b->m.size();
  return VD_OK;
}

int vd_batch_count_cells(const vd_batch* b, int index, size_t* n) {
  if (!b || !n || index < 0 || index >= (int)b->m.size()) return VD_EINVAL;
  if (!b->committed) return VD_ESTATE;
  *n = b->h_off[index + 1] - b->h_off[index];
  return VD_OK;
}

int vd_batch_get_generators(vd_batch* b, int index, double* xyz) {
  size_t n = 0;
  int r = vd_batch_count_cells(b, index, &n);
  if (r != VD_OK) return r;
  if (n) {
    B_CK(b, cudaMemcpyAsync(xyz, b->d_gen.p + 3 * (size_t)b->h_off[index], 3 * n * sizeof(double),
                            cudaMemcpyDeviceToHost, b->stream));
  }
  B_CK(b, cudaStreamSynchronize(b->stream));
  return VD_OK;
}

int vd_batch_get_summaries(vd_batch* b, int index, double* vol, double* centroid3, int32_t* n_faces) {
  size_t n = 0;
  int r = vd_batch_count_cells(b, index, &n);
  if (r != VD_OK) return r;
  if (!b->calculated) return bfail(b, VD_ESTATE, "calculate the batch first");
  const size_t o = b->h_off[index];
  cudaStream_t s = b->stream;
  if (n) {
    if (vol) B_CK(b, cudaMemcpyAsync(vol, b->d_vol.p + o, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (centroid3)
      B_CK(b, cudaMemcpyAsync(centroid3, b->d_cen.p + 3 * o, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (n_faces) B_CK(b, cudaMemcpyAsync(n_faces, b->d_nf.p + o, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  }
  B_CK(b, cudaStreamSynchronize(s));
  return VD_OK;
}

int vd_batch_total_cells(const vd_batch* b, size_t* n) {
  if (!b || !n) return VD_EINVAL;
  if (!b->committed) return VD_ESTATE;
  *n = b->h_off.empty() ? 0 : b->h_off.back();
  return VD_OK;
}

int vd_batch_timing(const vd_batch* b, float* ms) {
  if (!b || !ms) return VD_EINVAL;
  *ms = b->last_ms;
  return VD_OK;
}

int vd_batch_counters(const vd_batch* b, uint64_t* out8) {
  if (!b || !out8) return VD_EINVAL;
  for (int k = 0; k < kNumCounters; ++k) out8[k] = b->counters[k];
  return VD_OK;
}

int vd_batch_stream(vd_batch* b, void** stream) {
  if (!b || !stream) return VD_EINVAL;
  *stream = (void*)b->stream;
  return VD_OK;
}

}  // extern "C"
