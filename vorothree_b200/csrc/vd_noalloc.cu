// vd_noalloc.cu -- vd_calculate_noalloc: set_generators + calculate for a
// small tessellation without allocating any device memory.
//
// Who needs it: callers whose device memory is not theirs to allocate.  A
// plugin inside an application that reserves the GPU's memory up front and
// hands out fixed buffers, code that must go through a framework's memory
// pool, or a latency-critical loop that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree can trigger.  Such a caller passes its
// own device buffers for the generators and for the per-cell results; every
// intermediate buffer (bins, the bin-ordered generator copy, the search order,
// per-face slots, fallback lists and the large-capacity polytope storage)
// lives in one file-scope __device__ array of fixed size.
//
// Properties a caller must know:
//  * The scratch array (kNaBytes, about 8 MiB) is part of the library image:
//    every GPU that loads the library holds it until the process exits.
//  * All calls share that one array and it keeps the last call's contents.
//    Everything that must start at zero is cleared at the start of each call,
//    but two calls whose work overlaps on the GPU (different streams or
//    threads without ordering between them) race on the array and corrupt
//    each other's results.  Order such calls, e.g. one stream.
//  * The first call on a device looks up the device address of the array
//    (cudaGetSymbolAddress, with that device current) and caches it; make that
//    first call before any stream capture begins.
//  * Limits: at most kNaMaxGen generators, and a grid whose complete shell
//    search order fits kNaMaxOrder entries ((2nx+1)(2ny+1)(2nz+1) <= 68921,
//    e.g. 20x20x20).  Larger requests are rejected with VD_EINVAL.
//  * Cells are built by the shared-memory pass and, when they outgrow it, by
//    the large-capacity pass (2048 vertices, 512 faces); the regular entry
//    points send cells beyond that to a block-per-cell tier whose storage
//    (several MB per cell) this array does not hold.  Such a cell -- e.g. the
//    centre of generators on a sphere, adjacent to thousands of others --
//    makes the call return VD_EOVERFLOW, as does a total of more than
//    kNaPoolFaces faces in cells with more than 48 faces.
//  * No walls.  Every cell the call returns equals vd_tess_set_generators_device
//    + vd_tess_calculate bit for bit (same kernels, same arithmetic).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/voronoid_b200.h"
#include "vd_binning.cuh"
#include "vd_clip.cuh"
#include "vd_internal.h"
#include "vd_order.h"

using namespace vd;

namespace {

constexpr size_t kNaMaxGen = 8192;
constexpr size_t kNaMaxOrder = 68921;  // complete search order of a 20x20x20 grid
// (2nx+1)(2ny+1)(2nz+1) > 8 nx ny nz, so the order limit admits fewer than
// 68921 / 8 bins
constexpr size_t kNaMaxBins = 8616;
constexpr int kNaFout = 48;
constexpr size_t kNaPoolFaces = 16384;
constexpr int kNaBigWarps = 4;         // large-capacity pass: one block of 4 warps
constexpr size_t kNaSums = 64;

constexpr size_t al(size_t x) { return (x + 255) & ~size_t(255); }

// region offsets inside the scratch array
constexpr size_t kOffOrder = 0;
constexpr size_t kOffBinOf = kOffOrder + al(kNaMaxOrder * sizeof(Offset));
constexpr size_t kOffCounts = kOffBinOf + al(kNaMaxGen * 4);
constexpr size_t kOffStart = kOffCounts + al((kNaMaxBins + 1) * 4);
constexpr size_t kOffCursor = kOffStart + al((kNaMaxBins + 1) * 4);
constexpr size_t kOffIds = kOffCursor + al((kNaMaxBins + 1) * 4);
constexpr size_t kOffIdsTmp = kOffIds + al(kNaMaxGen * 4);
constexpr size_t kOffBigList = kOffIdsTmp + al(kNaMaxGen * 4);
constexpr size_t kOffSorted = kOffBigList + al(kNaMaxBins * 4);
constexpr size_t kOffNverts = kOffSorted + al(kNaMaxGen * sizeof(SortedGen));
constexpr size_t kOffStatus = kOffNverts + al(kNaMaxGen * 4);
constexpr size_t kOffFnb = kOffStatus + al(kNaMaxGen);
constexpr size_t kOffFarea = kOffFnb + al(kNaMaxGen * kNaFout * 4);
constexpr size_t kOffPoolOff = kOffFarea + al(kNaMaxGen * kNaFout * 8);
constexpr size_t kOffPoolFnb = kOffPoolOff + al(kNaMaxGen * 8);
constexpr size_t kOffPoolArea = kOffPoolFnb + al(kNaPoolFaces * 4);
constexpr size_t kOffList0 = kOffPoolArea + al(kNaPoolFaces * 8);
constexpr size_t kOffList1 = kOffList0 + al(kNaMaxGen * 4);
constexpr size_t kOffCtl = kOffList1 + al(kNaMaxGen * 4);        // u32[8]
constexpr size_t kOffCounters = kOffCtl + al(8 * 4);              // u64[kNumCounters]
constexpr size_t kOffPoolCursor = kOffCounters + al(kNumCounters * 8);
constexpr size_t kOffSums0 = kOffPoolCursor + al(8);
constexpr size_t kOffSums1 = kOffSums0 + al(kNaSums * 4);
constexpr size_t kOffBig = kOffSums1 + al(kNaSums * 4);
constexpr size_t kNaBytes = kOffBig + al(kNaBigWarps * sizeof(WarpPoly<BigCfg>));

static_assert((kNaMaxBins + 1 + kScanTile - 1) / kScanTile <= kNaSums, "scan sums");
static_assert(kNaMaxBins * 8 >= kNaMaxOrder, "every grid within the order limit fits the bin regions");

__device__ __align__(256) unsigned char g_vd_noalloc_scratch[kNaBytes];

struct NaDevice {
  bool ready = false;
  unsigned char* base = nullptr;
  ClipLaunchInfo info{};
  int sms = 0;
};

constexpr int kNaMaxDevices = 64;
std::mutex g_na_mutex;
NaDevice g_na_dev[kNaMaxDevices];

int na_fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  set_thread_error(buf);
  return code;
}

#define NA_CK(call)                                                                                 \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess) return na_fail(VD_ECUDA, "%s: %s", #call, cudaGetErrorString(e_));       \
  } while (0)

// Once per device, with that device current: the device address of the
// scratch array (host code must not use the symbol itself as a pointer) and
// the clip kernel's launch shape.
int na_setup(int dev, NaDevice** out) {
  if (dev < 0 || dev >= kNaMaxDevices) return na_fail(VD_EINVAL, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_na_mutex);
  NaDevice& d = g_na_dev[dev];
  if (!d.ready) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_vd_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return na_fail(VD_ECUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    e = clip_fp64_info(&d.info);
    if (e != cudaSuccess) return na_fail(VD_ECUDA, "clip kernel setup: %s", cudaGetErrorString(e));
    cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
    d.base = static_cast<unsigned char*>(p);
    d.ready = true;
  }
  *out = &d;
  return VD_OK;
}

template <typename T>
T* region(unsigned char* base, size_t off) {
  return reinterpret_cast<T*>(base + off);
}

int na_blocks(const NaDevice& d, size_t n, int threads) {
  const size_t want = (n + threads - 1) / threads;
  return (int)std::max<size_t>(1, std::min(want, (size_t)std::max(1, d.sms) * 16));
}

}  // namespace

extern "C" int vd_calculate_noalloc(const double bmin[3], const double bmax[3], int nx, int ny, int nz,
                                    const double* d_xyz, size_t n, double* d_volume, double* d_centroid3,
                                    int32_t* d_n_faces, void* stream) {
  if (!bmin || !bmax) return na_fail(VD_EINVAL, "null bounds");
  if (n > 0 && (!d_xyz || !d_volume || !d_centroid3 || !d_n_faces))
    return na_fail(VD_EINVAL, "null device buffer");
  if (n > kNaMaxGen)
    return na_fail(VD_EINVAL, "vd_calculate_noalloc: %zu generators exceed the limit of %zu", n, kNaMaxGen);
  if (nx <= 0 || ny <= 0 || nz <= 0) return na_fail(VD_EINVAL, "grid resolution must be positive");
  const double order_full = (2.0 * nx + 1) * (2.0 * ny + 1) * (2.0 * nz + 1);
  const size_t nbins = (size_t)nx * ny * nz;
  if (order_full <= (double)kNaMaxOrder && nbins > kNaMaxBins)  // excluded by the static_assert above
    return na_fail(VD_EINVAL, "vd_calculate_noalloc: grid %dx%dx%d has %zu bins, limit %zu", nx, ny, nz, nbins,
                   kNaMaxBins);
  if (order_full > (double)kNaMaxOrder)
    return na_fail(VD_EINVAL,
                   "vd_calculate_noalloc: grid %dx%dx%d needs %.0f search-order entries, limit %zu "
                   "((2nx+1)(2ny+1)(2nz+1) <= %zu, e.g. 20x20x20)",
                   nx, ny, nz, order_full, kNaMaxOrder, kNaMaxOrder);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return na_fail(VD_ECUDA, "no CUDA device");
  NaDevice* D = nullptr;
  int r = na_setup(dev, &D);
  if (r != VD_OK) return r;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char* base = D->base;

  // Algorithm3DGrid::new (algo_3d_grid.rs:47-95); the complete search order
  Grid g{};
  const int nn[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) {
    g.bmin[a] = bmin[a];
    g.bmax[a] = bmax[a];
    g.n[a] = nn[a];
    g.scale[a] = (double)nn[a] / (bmax[a] - bmin[a]);
    g.limit[a] = (double)nn[a] - 1e-5;
    g.cs[a] = 1.0 / g.scale[a];
  }
  std::vector<Offset> order;
  bool complete = false;
  double bound = 0.0;
  build_order(g, std::max(nx, std::max(ny, nz)), order, complete, bound);
  if (!complete || order.size() > kNaMaxOrder) return na_fail(VD_EINVAL, "search order does not fit");
  Offset* d_order = region<Offset>(base, kOffOrder);
  NA_CK(cudaMemcpyAsync(d_order, order.data(), order.size() * sizeof(Offset), cudaMemcpyHostToDevice, s));

  uint32_t* bin_of = region<uint32_t>(base, kOffBinOf);
  uint32_t* counts = region<uint32_t>(base, kOffCounts);
  uint32_t* start = region<uint32_t>(base, kOffStart);
  uint32_t* cursor = region<uint32_t>(base, kOffCursor);
  uint32_t* ids = region<uint32_t>(base, kOffIds);
  uint32_t* ids_tmp = region<uint32_t>(base, kOffIdsTmp);
  uint32_t* big_list = region<uint32_t>(base, kOffBigList);
  SortedGen* sorted = region<SortedGen>(base, kOffSorted);
  unsigned int* ctl = region<unsigned int>(base, kOffCtl);
  unsigned long long* counters = region<unsigned long long>(base, kOffCounters);
  unsigned long long* pool_cursor = region<unsigned long long>(base, kOffPoolCursor);
  uint32_t* sums0 = region<uint32_t>(base, kOffSums0);
  uint32_t* sums1 = region<uint32_t>(base, kOffSums1);

  // everything that must start at zero; the array keeps the last call's contents
  NA_CK(cudaMemsetAsync(counts, 0, (nbins + 1) * 4, s));
  NA_CK(cudaMemsetAsync(ctl, 0, 8 * 4, s));
  NA_CK(cudaMemsetAsync(counters, 0, kNumCounters * 8, s));
  NA_CK(cudaMemsetAsync(pool_cursor, 0, 8, s));

  // Algorithm3DGrid::set_generators (algo_3d_grid.rs:111-130) by counting sort
  if (n > 0) {
    k_bin_count<<<na_blocks(*D, n, 256), 256, 0, s>>>(d_xyz, n, g, bin_of, counts);
    NA_CK(cudaGetLastError());
  }
  {
    const size_t m = nbins + 1, nt = (m + kScanTile - 1) / kScanTile;
    k_scan_tiles<uint32_t, uint32_t><<<(unsigned)nt, kScanThreads, 0, s>>>(counts, start, m, sums0);
    NA_CK(cudaGetLastError());
    if (nt > 1) {
      k_scan_tiles<uint32_t, uint32_t><<<1, kScanThreads, 0, s>>>(sums0, sums1, nt, nullptr);
      NA_CK(cudaGetLastError());
      k_scan_add<uint32_t><<<(unsigned)nt, kScanThreads, 0, s>>>(start, m, sums1);
      NA_CK(cudaGetLastError());
    }
  }
  if (n > 0) {
    NA_CK(cudaMemcpyAsync(cursor, start, nbins * 4, cudaMemcpyDeviceToDevice, s));
    k_bin_scatter<<<na_blocks(*D, n, 256), 256, 0, s>>>(bin_of, n, cursor, ids);
    NA_CK(cudaGetLastError());
    k_bin_fix<<<na_blocks(*D, nbins, 256), 256, 0, s>>>(start, nbins, ids, big_list, ctl + 3);
    NA_CK(cudaGetLastError());
    k_bin_sort_big<<<std::max(1, D->sms), kBigSortThreads, 0, s>>>(start, big_list, ctl + 3, ids, ids_tmp);
    NA_CK(cudaGetLastError());
    k_gather_sorted<<<na_blocks(*D, n, 256), 256, 0, s>>>(ids, d_xyz, n, sorted);
    NA_CK(cudaGetLastError());
  }

  // Tessellation::calculate (tessellation.rs:213-230): the FP64 clip kernels
  TessDesc T;
  memset(&T, 0, sizeof(T));
  T.grid = g;
  T.nwalls = 0;
  T.order = d_order;
  T.norder = (int)order.size();
  T.order_complete = 1;
  T.order_bound = bound;
  T.gen = d_xyz;
  T.bin_of = bin_of;
  T.bin_start = start;
  T.sorted = sorted;
  T.ncells = (uint32_t)n;
  T.vol = d_volume;
  T.cen = d_centroid3;
  T.nfaces = d_n_faces;
  T.nverts = region<int32_t>(base, kOffNverts);
  T.fnb = region<int32_t>(base, kOffFnb);
  T.farea = region<double>(base, kOffFarea);
  T.status = region<uint8_t>(base, kOffStatus);
  T.fout = kNaFout;
  T.pool_fnb = region<int32_t>(base, kOffPoolFnb);
  T.pool_farea = region<double>(base, kOffPoolArea);
  T.pool_off = region<long long>(base, kOffPoolOff);
  T.pool_cursor = pool_cursor;
  T.pool_cap = (long long)kNaPoolFaces;

  if (n == 0) {
    NA_CK(cudaStreamSynchronize(s));
    return VD_OK;
  }
  uint32_t* list0 = region<uint32_t>(base, kOffList0);
  uint32_t* list1 = region<uint32_t>(base, kOffList1);
  WorkList W;
  memset(&W, 0, sizeof(W));
  W.items = nullptr;
  W.nitems = (uint32_t)n;
  W.cursor = ctl + 0;
  W.ovf_list = list0;
  W.ovf_count = ctl + 1;
  W.tab_list = list1;
  W.tab_count = ctl + 2;
  W.counters = counters;
  const int wpb = std::max(1, D->info.warps_per_block);
  const size_t warps_needed = (n + wpb - 1) / wpb;
  const int nblocks = (int)std::max<size_t>(
      1, std::min<size_t>(warps_needed, (size_t)D->sms * std::max(1, D->info.blocks_per_sm)));
  NA_CK(launch_clip_fp64_fast(T, W, nblocks, false, s));
  unsigned int h[3] = {0, 0, 0};
  NA_CK(cudaMemcpyAsync(h, ctl, sizeof(h), cudaMemcpyDeviceToHost, s));
  NA_CK(cudaStreamSynchronize(s));
  if (h[2] > 0) return na_fail(VD_EOVERFLOW, "search order exhausted on a complete table");
  if (h[1] > 0) {
    // polytopes that outgrew shared memory: the large-capacity pass over the
    // listed cells, its per-warp storage in the same scratch array
    const unsigned int novf = h[1];
    NA_CK(cudaMemsetAsync(ctl, 0, 3 * 4, s));
    W.items = list0;
    W.nitems = novf;
    W.ovf_list = list1;
    W.tab_list = list1;
    NA_CK(launch_clip_fp64_big(T, W, base + kOffBig, kNaBigWarps, s));
    unsigned long long used = 0;
    NA_CK(cudaMemcpyAsync(h, ctl, sizeof(h), cudaMemcpyDeviceToHost, s));
    NA_CK(cudaMemcpyAsync(&used, pool_cursor, sizeof(used), cudaMemcpyDeviceToHost, s));
    NA_CK(cudaStreamSynchronize(s));
    if (h[1] > 0 || h[2] > 0)
      return na_fail(VD_EOVERFLOW,
                     "vd_calculate_noalloc: %u cells exceed the large polytope capacity (2048 vertices, 512 faces); "
                     "the regular entry points build them",
                     h[1] + h[2]);
    if (used > kNaPoolFaces)
      return na_fail(VD_EOVERFLOW,
                     "vd_calculate_noalloc: cells with more than %d faces need %llu face slots, limit %zu", kNaFout,
                     used, kNaPoolFaces);
  }
  return VD_OK;
}
