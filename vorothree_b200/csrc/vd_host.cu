// vd_host.cu -- host side of the C ABI (include/voronoid_b200.h).
//
// A vd_tess owns one CUDA stream and every device buffer of one
// tessellation: the generators, their bins, the search order, and the
// per-cell outputs.  Data stays resident in HBM between calls; the host only
// sees it through the result getters.
//
// Compiled with -fmad=false: the host-side wall normalisation and the
// device-side wall tests and bin indices must round exactly like the
// reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/voronoid_b200.h"
#include "vd_binning.cuh"
#include "vd_wall.cuh"
#include "vd_internal.h"
#include "vd_order.h"

using namespace vd;

namespace {

thread_local std::string g_create_error;
// grids whose complete search order has at most this many entries get the
// complete table; larger ones start truncated (k = 8) and grow on demand
constexpr int kCompleteOrderMax = 1 << 15;
// longest truncated search order (in bins per axis) chosen from the density
// before a first pass; longer ones come only from cells that ran off it
constexpr int kMaxInitialOrder = 32;
// blocks of the huge tier (each holds its cell's polytope in global memory)
constexpr int kHugeBlocksMax = 64;
// face capacities of the tiers whose cells can have more faces than the
// per-cell slots hold (medium, large, huge): their faces go to the pool
constexpr long long kMedFaces = 112, kBigFaces = 512, kHugeFaces = 32767;
// cells the slot layout hands off, from which they go through the
// full-rewrite first tier before the medium tier
constexpr int kFullHandoffMin = 256;
// kernels this library has launched in this process (all handles)
std::atomic<unsigned long long> g_launches{0};

// The library's memory pool on each device: stream-ordered allocations that
// stay reserved for the process once freed (release threshold = max), so a
// buffer that grows reuses memory without going back to the driver.
cudaError_t lib_pool(cudaMemPool_t* out) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  auto it = pools.find(dev);
  if (it != pools.end()) {
    *out = it->second;
    return cudaSuccess;
  }
  cudaMemPoolProps props;
  memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool;
  e = cudaMemPoolCreate(&pool, &props);
  if (e != cudaSuccess) return e;
  uint64_t keep = ~0ull;
  e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  if (e != cudaSuccess) return e;
  pools[dev] = pool;
  *out = pool;
  return cudaSuccess;
}

// A device buffer that only grows.  Allocation is stream-ordered, on the
// handle's stream from the library's pool: growing one handle's buffers
// never synchronises the device (as cudaFree does), so handles serving
// concurrent requests do not stall each other.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;  // elements
  cudaStream_t s = nullptr;  // stream of the last allocation (frees are ordered on it)
  cudaError_t ensure(size_t n, cudaStream_t stream) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    cap = 0;
    s = stream;
    if (vd::injected_alloc_failure()) return cudaErrorMemoryAllocation;
    const size_t want = std::max<size_t>(n, 1);
    cudaMemPool_t pool;
    cudaError_t e = lib_pool(&pool);
    if (e != cudaSuccess) return e;
    e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), want * sizeof(T), pool, stream);
    if (e == cudaSuccess) cap = want;
    else p = nullptr;
    return e;
  }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    cap = 0;
  }
};

// offsets of the small device-side control block
enum : int {
  kCtlCursor = 0,
  kCtlOvfCount,
  kCtlTabCount,
  kCtlBigCount,
  kCtlWords = 8,
};

}  // namespace

namespace {
// an axis normalised as CylinderGeometry/ConeGeometry/TorusGeometry::new do
// (wall_3d.rs:124-128, 194-198, 285-289)
static void unit_axis(const double axis[3], double out[3]) {
  const double len = std::sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
  if (len == 0.0) {
    out[0] = 0.0;
    out[1] = 0.0;
    out[2] = 1.0;
  } else {
    for (int a = 0; a < 3; ++a) out[a] = axis[a] / len;
  }
}
}  // namespace

namespace vd {
void set_thread_error(const char* msg) { g_create_error = msg; }

namespace {
std::atomic<int> g_fail_allocs{0};
}

bool injected_alloc_failure() {
  int k = g_fail_allocs.load();
  while (k > 0)
    if (g_fail_allocs.compare_exchange_weak(k, k - 1)) return true;
  return false;
}

void set_scratch_caps(vd_tess* t, size_t big_warps, size_t huge_blocks);

cudaError_t reserve_pool(size_t bytes, cudaStream_t s) {
  cudaMemPool_t pool;
  cudaError_t e = lib_pool(&pool);
  if (e != cudaSuccess || bytes == 0) return e;
  void* p = nullptr;
  e = cudaMallocFromPoolAsync(&p, bytes, pool, s);
  if (e != cudaSuccess) return e;
  e = cudaFreeAsync(p, s);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}
}  // namespace vd

namespace vd {
bool wall_from_desc(const vd_wall_desc& d, Wall* w, std::vector<double>* planes, std::string* err) {
  memset(w, 0, sizeof(*w));
  w->kind = d.kind;
  w->id = d.id;
  if (d.id > VD_WALL_ID_MAX) {
    *err = "Wall ID must be <= " + std::to_string(VD_WALL_ID_MAX);
    return false;
  }
  for (int a = 0; a < 3; ++a) w->a[a] = d.a[a];
  switch (d.kind) {
    case kWallPlane: {  // PlaneGeometry::new (wall_3d.rs:23-27)
      const double len = std::sqrt(d.n[0] * d.n[0] + d.n[1] * d.n[1] + d.n[2] * d.n[2]);
      if (len == 0.0) w->n[2] = 1.0;
      else
        for (int a = 0; a < 3; ++a) w->n[a] = d.n[a] / len;
      return true;
    }
    case kWallSphere:
      w->r = d.r;
      return true;
    case kWallCylinder:
    case kWallCone:
    case kWallTorus:
      unit_axis(d.n, w->n);
      w->r = d.r;
      w->r2 = d.r2;
      if (d.kind == kWallCone) {
        w->ca = std::cos(d.r);
        w->sa = std::sin(d.r);
        w->ta = std::tan(d.r);
      }
      return true;
    case kWallPolyhedron:
      if (d.nplanes < 0 || (d.nplanes > 0 && (!d.points || !d.normals))) {
        *err = "bad polyhedron planes";
        return false;
      }
      w->np = d.nplanes;
      w->p0 = (int)(planes->size() / 6);
      for (int k = 0; k < d.nplanes; ++k) {
        for (int a = 0; a < 3; ++a) planes->push_back(d.points[3 * k + a]);
        for (int a = 0; a < 3; ++a) planes->push_back(d.normals[3 * k + a]);
      }
      return true;
    default:
      *err = "unknown wall kind " + std::to_string(d.kind);
      return false;
  }
}
}  // namespace vd

// the block-per-cell tier's width: tessellations of at most this many cells
// run it with 16-warp blocks (on the slot layout 16 warps win at every size
// measured, 1,000 to 20,000 generators on a sphere), larger ones with 32
constexpr int kHugeNarrowDefault = 1 << 30;
// the slot layout's register budget: 7 blocks of four warps per SM for FP64
// (the autotuner's choice for uniform input from 2^16 cells and clustered
// from 2^18: 1 M uniform cells 32.5 ms against 33.5 at 6 and 33.7 at 5), 6
// for the mixed path (whose FP32 copies spill more at 7: 0.80 against 0.86 of
// FP64 on 1 M uniform cells)
constexpr int kFastMinbDefault = 7;
constexpr int kFastMinbDefaultMixed = 6;
// the walk's batched plane tests after a run of clips that change nothing
// (-1: off)
constexpr int kNoopRunDefault = -1;

struct vd_tess {
  std::string err;
  int device = 0;
  cudaStream_t stream = nullptr;
  Grid grid{};
  std::vector<Wall> walls;
  std::vector<double> planes;  // plane table of convex-polyhedron walls (6 doubles each)
  DevBuf<double> d_planes;
  int precision = VD_PREC_FP64;
  bool instrument = false;  // run the counting kernel variant

  // search order
  int order_k = 0;
  bool order_complete = false;
  double order_bound = 0.0;
  int norder = 0;
  DevBuf<Offset> d_order;

  // generators and bins
  size_t ngen = 0;
  size_t nbins = 0;
  DevBuf<double> d_gen, d_in, d_tmp3;
  DevBuf<uint32_t> d_flags, d_pos;
  DevBuf<uint32_t> d_bin_of, d_bin_count, d_bin_start, d_cursor, d_ids, d_ids_tmp, d_big_list;
  DevBuf<SortedGen> d_sorted;
  DevBuf<uint32_t> d_occ;   // bin occupancy bits (sparse grids)
  bool occ_valid = false;

  // outputs
  size_t ncells = 0;
  bool calculated = false;
  int fout = 48;
  DevBuf<double> d_vol, d_cen, d_pool_area, d_csr_area;
  DevBuf<int32_t> d_nf, d_nv, d_fnb, d_pool_fnb, d_csr_ids;
  DevBuf<double> d_farea;
  DevBuf<uint8_t> d_status;
  DevBuf<long long> d_pool_off, d_csr_off, d_nf64;
  bool csr_valid = false;
  long long csr_total = 0;
  size_t range_begin = 0, range_end = 0;  // cells computed by the last calculate
  // ... of which those with ((id - range_begin) / range_chunk) % range_stride == range_phase
  size_t range_chunk = 1, range_stride = 1, range_phase = 0;

  // control
  DevBuf<unsigned int> d_ctl;
  DevBuf<unsigned long long> d_counters, d_pool_cursor;
  DevBuf<uint32_t> d_list[3];
  DevBuf<unsigned char> d_big, d_huge;
  size_t big_warps = 0, huge_blocks = 0;
  // most warps / blocks the large and huge tiers may hold scratch for (the
  // persistent kernels take any number; a server bounds a slot's scratch)
  size_t big_warps_cap = (size_t)-1, huge_blocks_cap = (size_t)-1;
  long long pool_cap = 0;
  // the pool cursor as the host last read it (after every clip pass)
  unsigned long long pool_used = 0;

  // scan scratch
  std::vector<DevBuf<uint32_t>> scan32;
  std::vector<DevBuf<long long>> scan64;

  // calculate_sealed / prune_boundaries
  bool sealed = false;
  DevBuf<int32_t> d_s_nf, d_s_fnb, d_s_pool_fnb;
  DevBuf<long long> d_s_pool_off;
  DevBuf<uint32_t> d_s_mask, d_c_mask, d_sel;
  DevBuf<SealLogRec> d_seal_rec;
  DevBuf<PruneRec> d_prune_rec;
  DevBuf<PrunePos> d_prune_posrec;
  DevBuf<unsigned int> d_rec_cursor;
  DevBuf<int32_t> d_lcnt, d_lpcnt;
  DevBuf<long long> d_loff, d_lpoff;
  DevBuf<int32_t> d_seal_log, d_prune_log;
  DevBuf<double> d_prune_pos;
  size_t nseal = 0, nprune = 0, nprune_pos = 0;

  // export buffers for get_cell
  DevBuf<double> d_ex_v;
  DevBuf<uint32_t> d_ex_fc, d_ex_fi;
  DevBuf<int32_t> d_ex_fn, d_ex_sizes;
  // bulk export (vd_tess_export_cells)
  DevBuf<uint32_t> d_bx_items, d_bx_fc, d_bx_fi;
  DevBuf<int32_t> d_bx_sizes, d_bx_fn;
  DevBuf<long long> d_bx_off;
  DevBuf<double> d_bx_v;

  // instrumentation
  cudaEvent_t ev[8] = {};
  float timings[4] = {0, 0, 0, 0};
  unsigned long long counters[kNumCounters] = {};
  unsigned long long fallback[2] = {0, 0};
  ClipLaunchInfo info64{}, infomx{}, infomed{};
  ClipLaunchInfo infosp64[3]{}, infospmx[3]{};  // slot layout at 5, 6, 7 blocks per SM
  int fast_layout = VD_FAST_SLOTS;
  int fast_minb = 0;  // 0: the precision's default (fast_minb_for)
  int huge_direct_max = 64;
  int huge_blocks_max = 64;
  int huge_narrow_max = kHugeNarrowDefault;
  int noop_run = kNoopRunDefault;
  int num_sms = 0;
};

namespace {

int fail(vd_tess* t, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (t) t->err = buf;
  else g_create_error = buf;
  return code;
}

#define VD_CK(t, call)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return fail((t), e_ == cudaErrorMemoryAllocation ? VD_ENOMEM : VD_ECUDA, "%s: %s (%s:%d)", \
                  #call, cudaGetErrorString(e_), __FILE__, __LINE__);                            \
  } while (0)

int grid_blocks(const vd_tess* t, size_t n, int threads) {
  const size_t want = (n + threads - 1) / threads;
  const size_t cap = (size_t)std::max(1, t->num_sms) * 16;
  return (int)std::max<size_t>(1, std::min(want, cap));
}

// exclusive scan of n values of `in` into out[0..n); out must hold n+1 and
// gets the total at out[n] when `with_total`.
template <typename Tin, typename T>
int scan_excl(vd_tess* t, const Tin* in, T* out, size_t n, std::vector<DevBuf<T>>& pool, int level = 0) {
  if (n == 0) return VD_OK;
  const size_t nt = (n + kScanTile - 1) / kScanTile;
  if ((int)pool.size() <= level) pool.resize(level + 1);
  VD_CK(t, pool[level].ensure(nt + 1, t->stream));
  T* sums = pool[level].p;
  k_scan_tiles<Tin, T><<<(unsigned)nt, kScanThreads, 0, t->stream>>>(in, out, n, sums);
  g_launches++;
  VD_CK(t, cudaGetLastError());
  if (nt > 1) {
    // scan the tile sums in place (needs its own level of scratch)
    if ((int)pool.size() <= level + 1) pool.resize(level + 2);
    VD_CK(t, pool[level + 1].ensure(nt + 1, t->stream));
    T* sscan = pool[level + 1].p;
    int r = scan_excl<T, T>(t, sums, sscan, nt, pool, level + 2);
    if (r != VD_OK) return r;
    k_scan_add<T><<<(unsigned)nt, kScanThreads, 0, t->stream>>>(out, n, sscan);
    g_launches++;
    VD_CK(t, cudaGetLastError());
  }
  return VD_OK;
}

int upload_order(vd_tess* t, int k) {
  std::vector<Offset> h;
  bool complete;
  double bound;
  build_order(t->grid, k, h, complete, bound);
  VD_CK(t, t->d_order.ensure(h.size(), t->stream));
  VD_CK(t, cudaMemcpyAsync(t->d_order.p, h.data(), h.size() * sizeof(Offset), cudaMemcpyHostToDevice, t->stream));
  VD_CK(t, cudaStreamSynchronize(t->stream));
  t->order_k = k;
  t->order_complete = complete;
  t->order_bound = bound;
  t->norder = (int)h.size();
  return VD_OK;
}

WallSet wallset(const vd_tess* t) {
  WallSet ws;
  memset(&ws, 0, sizeof(ws));
  ws.n = (int)t->walls.size();
  for (int i = 0; i < ws.n; ++i) ws.w[i] = t->walls[i];
  ws.planes = t->d_planes.p;
  return ws;
}

// bins per generator from which the walk tests bins through the occupancy
// bit map: on such sparse grids most bins it reaches are empty, and the bit
// map (1/32 of the bin table) stays in L2 where the table does not
constexpr size_t kOccupancyBinsPerGen = 8;

// the occupancy bit map of the current bins, on sparse grids
int build_occupancy(vd_tess* t) {
  const size_t nb = t->nbins;
  t->occ_valid = false;
  if (nb < kOccupancyBinsPerGen * std::max<size_t>(t->ngen, 1)) return VD_OK;
  VD_CK(t, t->d_occ.ensure((nb + 31) / 32, t->stream));
  k_bin_occupancy<<<grid_blocks(t, (nb + 31) / 32, 256), 256, 0, t->stream>>>(t->d_bin_start.p, nb, t->d_occ.p);
  g_launches++;
  VD_CK(t, cudaGetLastError());
  t->occ_valid = true;
  return VD_OK;
}

// Algorithm3DGrid::set_generators on the device: bin index, counting sort
// with members in ascending id order, then the bin-ordered copy.
int rebin(vd_tess* t) {
  const size_t n = t->ngen, nb = t->nbins;
  cudaStream_t s = t->stream;
  VD_CK(t, t->d_bin_of.ensure(n, t->stream));
  VD_CK(t, t->d_bin_count.ensure(nb + 1, t->stream));
  VD_CK(t, t->d_bin_start.ensure(nb + 1, t->stream));
  VD_CK(t, t->d_cursor.ensure(nb + 1, t->stream));
  VD_CK(t, t->d_ids.ensure(n, t->stream));
  VD_CK(t, t->d_ids_tmp.ensure(n, t->stream));
  VD_CK(t, t->d_big_list.ensure(nb, t->stream));
  VD_CK(t, t->d_sorted.ensure(n, t->stream));
  VD_CK(t, t->d_ctl.ensure(kCtlWords, t->stream));
  VD_CK(t, cudaMemsetAsync(t->d_bin_count.p, 0, (nb + 1) * sizeof(uint32_t), s));
  VD_CK(t, cudaMemsetAsync(t->d_ctl.p + kCtlBigCount, 0, sizeof(unsigned int), s));
  if (n > 0) {
    k_bin_count<<<grid_blocks(t, n, 256), 256, 0, s>>>(t->d_gen.p, n, t->grid, t->d_bin_of.p, t->d_bin_count.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
  }
  int r = scan_excl<uint32_t, uint32_t>(t, t->d_bin_count.p, t->d_bin_start.p, nb + 1, t->scan32);
  if (r != VD_OK) return r;
  if (n > 0) {
    VD_CK(t, cudaMemcpyAsync(t->d_cursor.p, t->d_bin_start.p, nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    k_bin_scatter<<<grid_blocks(t, n, 256), 256, 0, s>>>(t->d_bin_of.p, n, t->d_cursor.p, t->d_ids.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
    k_bin_fix<<<grid_blocks(t, nb, 256), 256, 0, s>>>(t->d_bin_start.p, nb, t->d_ids.p, t->d_big_list.p,
                                                       t->d_ctl.p + kCtlBigCount);
    g_launches++;
    VD_CK(t, cudaGetLastError());
    k_bin_sort_big<<<std::max(1, t->num_sms), kBigSortThreads, 0, s>>>(
        t->d_bin_start.p, t->d_big_list.p, t->d_ctl.p + kCtlBigCount, t->d_ids.p, t->d_ids_tmp.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
    k_gather_sorted<<<grid_blocks(t, n, 256), 256, 0, s>>>(t->d_ids.p, t->d_gen.p, n, t->d_sorted.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
  }
  r = build_occupancy(t);
  if (r != VD_OK) return r;
  t->calculated = false;
  t->csr_valid = false;
  return VD_OK;
}

// keep the rows of d_in inside every wall (stable), into d_gen
int filter_into_gen(vd_tess* t, const double* d_src, size_t n, size_t* n_kept) {
  cudaStream_t s = t->stream;
  if (t->walls.empty()) {
    VD_CK(t, t->d_gen.ensure(3 * n, t->stream));
    if (n && d_src != t->d_gen.p)
      VD_CK(t, cudaMemcpyAsync(t->d_gen.p, d_src, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    t->ngen = n;
    if (n_kept) *n_kept = n;
    return VD_OK;
  }
  VD_CK(t, t->d_flags.ensure(n + 1, t->stream));
  VD_CK(t, t->d_pos.ensure(n + 1, t->stream));
  VD_CK(t, t->d_tmp3.ensure(3 * n, t->stream));
  if (n) {
    k_wall_flags<<<grid_blocks(t, n, 256), 256, 0, s>>>(d_src, n, wallset(t), t->d_flags.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
  }
  VD_CK(t, cudaMemsetAsync(t->d_flags.p + n, 0, sizeof(uint32_t), s));
  int r = scan_excl<uint32_t, uint32_t>(t, t->d_flags.p, t->d_pos.p, n + 1, t->scan32);
  if (r != VD_OK) return r;
  if (n) {
    k_compact3<<<grid_blocks(t, n, 256), 256, 0, s>>>(d_src, n, t->d_flags.p, t->d_pos.p, t->d_tmp3.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
  }
  uint32_t kept = 0;
  VD_CK(t, cudaMemcpyAsync(&kept, t->d_pos.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaStreamSynchronize(s));
  std::swap(t->d_gen, t->d_tmp3);
  t->ngen = kept;
  if (n_kept) *n_kept = kept;
  return VD_OK;
}

TessDesc make_desc(vd_tess* t) {
  TessDesc T;
  memset(&T, 0, sizeof(T));
  T.grid = t->grid;
  T.nwalls = (int)t->walls.size();
  for (int i = 0; i < T.nwalls; ++i) T.walls[i] = t->walls[i];
  T.planes = t->d_planes.p;
  T.order = t->d_order.p;
  T.norder = t->norder;
  T.order_complete = t->order_complete ? 1 : 0;
  T.order_bound = t->order_bound;
  T.gen = t->d_gen.p;
  T.bin_of = t->d_bin_of.p;
  T.bin_start = t->d_bin_start.p;
  T.occ = t->occ_valid ? t->d_occ.p : nullptr;
  T.noop_run = t->noop_run > 0 ? t->noop_run : 0;
  T.sorted = t->d_sorted.p;
  T.ncells = (uint32_t)t->ngen;
  T.vol = t->d_vol.p;
  T.cen = t->d_cen.p;
  T.nfaces = t->d_nf.p;
  T.nverts = t->d_nv.p;
  T.fnb = t->d_fnb.p;
  T.farea = t->d_farea.p;
  T.status = t->d_status.p;
  T.fout = t->fout;
  T.pool_fnb = t->d_pool_fnb.p;
  T.pool_farea = t->d_pool_area.p;
  T.pool_off = t->d_pool_off.p;
  T.pool_cursor = t->d_pool_cursor.p;
  T.pool_cap = t->pool_cap;
  return T;
}

int ensure_outputs(vd_tess* t, size_t n) {
  VD_CK(t, t->d_vol.ensure(n, t->stream));
  VD_CK(t, t->d_cen.ensure(3 * n, t->stream));
  VD_CK(t, t->d_nf.ensure(n, t->stream));
  VD_CK(t, t->d_nv.ensure(n, t->stream));
  VD_CK(t, t->d_fnb.ensure(n * (size_t)t->fout, t->stream));
  VD_CK(t, t->d_farea.ensure(n * (size_t)t->fout, t->stream));
  VD_CK(t, t->d_status.ensure(n, t->stream));
  VD_CK(t, t->d_pool_off.ensure(n, t->stream));
  VD_CK(t, t->d_ctl.ensure(kCtlWords, t->stream));
  VD_CK(t, t->d_counters.ensure(kNumCounters, t->stream));
  VD_CK(t, t->d_pool_cursor.ensure(1, t->stream));
  for (int k = 0; k < 3; ++k) VD_CK(t, t->d_list[k].ensure(n, t->stream));
  return VD_OK;
}

int ensure_big(vd_tess* t, size_t cells) {
  // enough warps to spread the listed cells, capped to bound the scratch
  // the big kernel runs 4 warps per block: scratch covers whole blocks
  size_t want = std::min<size_t>(std::max<size_t>(cells, 1), (size_t)std::max(1, t->num_sms) * 4);
  want = std::min(want, std::max<size_t>(t->big_warps_cap, 4));
  want = (want + 3) / 4 * 4;
  if (t->big_warps < want) {
    VD_CK(t, t->d_big.ensure(want * t->info64.big_scratch_per_warp, t->stream));
    t->big_warps = want;
  }
  return VD_OK;
}

// Most faces one cell can have in a tier of face capacity fcap: a face per
// other generator, per box side and per wall plane; seal clips add at most
// one more face per other generator.
long long faces_bound(const vd_tess* t, long long fcap, bool seal) {
  long long planes = 0;
  for (const Wall& w : t->walls) planes += w.kind == kWallPolyhedron ? w.np : 1;
  const long long others = t->ngen > 0 ? (long long)t->ngen - 1 : 0;
  return std::min(fcap, (seal ? 2 : 1) * others + 6 + planes);
}

// The face pool holds the face slots of cells with more faces than the
// per-cell slots.  Before a pass of a tier that can finish such cells, the
// pool is grown to hold every cell of the pass at the tier's largest face
// count beyond what earlier passes used, so a finished cell always gets its
// slots; the used part is kept when the pool grows.
int ensure_pool(vd_tess* t, size_t cells, long long faces_per_cell) {
  const unsigned long long need = t->pool_used + (unsigned long long)cells * (unsigned long long)faces_per_cell;
  if ((long long)need <= t->pool_cap) return VD_OK;
  const long long cap = std::max<long long>({(long long)need, 2 * t->pool_cap, 1LL << 20});
  DevBuf<int32_t> fnb;
  DevBuf<double> area;
  VD_CK(t, fnb.ensure((size_t)cap, t->stream));
  VD_CK(t, area.ensure((size_t)cap, t->stream));
  if (t->pool_used > 0) {
    VD_CK(t, cudaMemcpyAsync(fnb.p, t->d_pool_fnb.p, t->pool_used * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                             t->stream));
    VD_CK(t, cudaMemcpyAsync(area.p, t->d_pool_area.p, t->pool_used * sizeof(double), cudaMemcpyDeviceToDevice,
                             t->stream));
  }
  t->d_pool_fnb.release();
  t->d_pool_area.release();
  t->d_pool_fnb = fnb;
  t->d_pool_area = area;
  fnb.p = nullptr;
  area.p = nullptr;
  t->pool_cap = cap;
  return VD_OK;
}

int ensure_huge(vd_tess* t, size_t cells) {
  // a few blocks: each holds a multi-megabyte polytope in global memory
  const size_t want = std::min<size_t>(std::min<size_t>(std::max<size_t>(cells, 1), (size_t)t->huge_blocks_max),
                                       std::max<size_t>(t->huge_blocks_cap, 1));
  if (t->huge_blocks != want) {
    VD_CK(t, t->d_huge.ensure(want * clip_huge_scratch_per_block(), t->stream));
    t->huge_blocks = want;
  }
  return VD_OK;
}

// the slot layout's blocks per SM in force: the tuning setting, else the
// precision's default
int fast_minb_for(const vd_tess* t) {
  if (t->fast_minb) return t->fast_minb;
  return t->precision == VD_PREC_MIXED ? kFastMinbDefaultMixed : kFastMinbDefault;
}

// one pass of the clip kernel over `items` (nullptr = all cells in bin order);
// tier 0 = first tier (shared memory, the handle's layout), -1 = first tier on
// the full-rewrite layout (the slot layout's hand-offs), 1 = medium capacity,
// 2 = large capacity, 3 = huge capacity
int clip_pass(vd_tess* t, int tier, const uint32_t* items, uint32_t nitems, uint32_t* ovf_list,
              uint32_t* tab_list, const WorkList* extra = nullptr) {
  cudaStream_t s = t->stream;
  VD_CK(t, cudaMemsetAsync(t->d_ctl.p, 0, 3 * sizeof(unsigned int), s));
  WorkList W;
  memset(&W, 0, sizeof(W));
  if (extra) W = *extra;
  W.items = items;
  W.nitems = nitems;
  W.cursor = t->d_ctl.p + kCtlCursor;
  W.ovf_list = ovf_list;
  W.ovf_count = t->d_ctl.p + kCtlOvfCount;
  W.tab_list = tab_list;
  W.tab_count = t->d_ctl.p + kCtlTabCount;
  W.counters = t->d_counters.p;
  if (tier >= 1) {
    const long long fcap = tier == 1 ? kMedFaces : (tier == 2 ? kBigFaces : kHugeFaces);
    int r = ensure_pool(t, nitems, faces_bound(t, fcap, false));
    if (r != VD_OK) return r;
  }
  TessDesc T = make_desc(t);
  if (tier == 1) {
    const int nblocks = (int)std::max<size_t>(
        1, std::min<size_t>((nitems + 1) / 2, (size_t)t->num_sms * std::max(1, t->infomed.blocks_per_sm)));
    VD_CK(t, launch_clip_med(T, W, nblocks, t->instrument, s, t->noop_run > 0));
    g_launches++;
  } else if (tier <= 0) {
    const bool mixed = t->precision == VD_PREC_MIXED;
    // the slot layout cannot export a polytope in the reference's vertex
    // order: get_cell's rebuild runs the full-rewrite kernel
    const bool slots = tier == 0 && t->fast_layout == VD_FAST_SLOTS && !W.ex_verts;
    const int minb = fast_minb_for(t);
    const int mv = minb - 5;
    const ClipLaunchInfo& li =
        slots ? (mixed ? t->infospmx[mv] : t->infosp64[mv]) : (mixed ? t->infomx : t->info64);
    const size_t warps_needed = (nitems + li.warps_per_block - 1) / li.warps_per_block;
    const int nblocks = (int)std::max<size_t>(
        1, std::min<size_t>(warps_needed, (size_t)t->num_sms * std::max(1, li.blocks_per_sm)));
    if (slots)
      VD_CK(t, launch_clip_sparse(T, W, nblocks, t->instrument, mixed, minb, t->noop_run > 0, s));
    else
      VD_CK(t, mixed ? launch_clip_mixed_fast(T, W, nblocks, t->instrument, s)
                     : launch_clip_fp64_fast(T, W, nblocks, t->instrument, s, t->noop_run > 0));
    g_launches++;
  } else if (tier == 2) {
    int r = ensure_big(t, nitems);
    if (r != VD_OK) return r;
    T = make_desc(t);
    VD_CK(t, launch_clip_fp64_big(T, W, t->d_big.p, (int)t->big_warps, s, t->noop_run > 0));
    g_launches++;
  } else {
    int r = ensure_huge(t, nitems);
    if (r != VD_OK) return r;
    T = make_desc(t);
    VD_CK(t, launch_clip_fp64_huge(T, W, t->d_huge.p, (int)t->huge_blocks,
                                   T.ncells <= (uint32_t)t->huge_narrow_max, s));
    g_launches++;
  }
  return VD_OK;
}

// the pass's overflow and table counts, and the face pool's cursor; a cell
// whose faces found no room in the pool is an error (ensure_pool sizes the
// pool so that this cannot happen)
int read_ctl(vd_tess* t, unsigned int* ovf, unsigned int* tab) {
  unsigned int h[3];
  VD_CK(t, cudaMemcpyAsync(h, t->d_ctl.p, sizeof(h), cudaMemcpyDeviceToHost, t->stream));
  VD_CK(t, cudaMemcpyAsync(&t->pool_used, t->d_pool_cursor.p, sizeof(t->pool_used), cudaMemcpyDeviceToHost,
                           t->stream));
  VD_CK(t, cudaStreamSynchronize(t->stream));
  *ovf = h[kCtlOvfCount];
  *tab = h[kCtlTabCount];
  if ((long long)t->pool_used > t->pool_cap)
    return fail(t, VD_EOVERFLOW, "face pool overflow: %llu face slots needed, %lld available", t->pool_used,
                t->pool_cap);
  return VD_OK;
}

// cells of [begin, end) whose chunk index (id - begin) / chunk is phase
// modulo stride
size_t strided_count(const size_t* range) {
  const size_t len = range[1] - range[0], chunk = range[2], stride = range[3], phase = range[4];
  const size_t period = chunk * stride, full = len / period, rest = len % period;
  const size_t lo = phase * chunk;
  return full * chunk + (rest > lo ? std::min(chunk, rest - lo) : 0);
}

bool cell_computed(const vd_tess* t, size_t i) {
  return i >= t->range_begin && i < t->range_end &&
         ((i - t->range_begin) / t->range_chunk) % t->range_stride == t->range_phase;
}

// Runs the fast pass over all cells, then resolves the cells it could not
// finish: a longer search order for cells that walked off a truncated one,
// the large-capacity pass for polytopes that outgrew shared memory.
//
// only_cell: compute that one cell (get_cell's export).  range: compute the
// cells with ids in [range[0], range[1]) and clear the others.
int run_calculate(vd_tess* t, const WorkList* extra = nullptr, const uint32_t* only_cell = nullptr,
                  const size_t* range = nullptr) {
  // range: {begin, end, chunk, stride, phase} -- the cells with ids in
  // [begin, end) and ((id - begin) / chunk) % stride == phase
  cudaStream_t s = t->stream;
  const size_t n = t->ngen;
  int r = ensure_outputs(t, n);
  if (r != VD_OK) return r;
  VD_CK(t, cudaMemsetAsync(t->d_counters.p, 0, kNumCounters * sizeof(unsigned long long), s));
  if (!only_cell) {
    // a new tessellation: the pool starts empty and no cell has pooled faces
    // (-1); one cell rebuilt for get_cell appends to the pool instead, so the
    // other cells' pooled faces stay where they are
    VD_CK(t, cudaMemsetAsync(t->d_pool_cursor.p, 0, sizeof(unsigned long long), s));
    VD_CK(t, cudaMemsetAsync(t->d_pool_off.p, 0xFF, n * sizeof(long long), s));
    t->pool_used = 0;
  }
  t->fallback[0] = t->fallback[1] = 0;
  // A truncated search order long enough for the generator density before
  // the first pass: on sparse grids (many bins per generator) cells walk past
  // a short table and would be rerun from scratch with a longer one.  The walk
  // reaches about twice the neighbour spacing, ~4x the spacing in bins.
  if (!t->order_complete && !only_cell && n > 0) {
    const double spacing = std::cbrt((double)t->nbins / (double)n);
    const int k0 = std::min(kMaxInitialOrder, (int)std::ceil(4.0 * spacing) + 2);
    if (k0 > t->order_k) {
      r = upload_order(t, k0);
      if (r != VD_OK) return r;
    }
  }
  VD_CK(t, cudaEventRecord(t->ev[2], s));
  uint32_t* in_list = nullptr;
  uint32_t nin = only_cell ? 1u : (uint32_t)n;
  if (only_cell) {
    VD_CK(t, cudaMemcpyAsync(t->d_list[2].p, only_cell, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    in_list = t->d_list[2].p;
  } else if (range && (range[0] > 0 || range[1] < n || range[3] > 1)) {
    VD_CK(t, t->d_flags.ensure(n + 1, t->stream));
    VD_CK(t, t->d_pos.ensure(n + 1, t->stream));
    if (n) {
      k_clear_cells<<<grid_blocks(t, n, 256), 256, 0, s>>>(n, t->d_vol.p, t->d_cen.p, t->d_nf.p, t->d_nv.p);
      g_launches++;
      VD_CK(t, cudaGetLastError());
      k_range_flags<<<grid_blocks(t, n, 256), 256, 0, s>>>(t->d_sorted.p, n, (long long)range[0],
                                                           (long long)range[1], (long long)range[2],
                                                           (long long)range[3], (long long)range[4], t->d_flags.p);
      g_launches++;
      VD_CK(t, cudaGetLastError());
    }
    VD_CK(t, cudaMemsetAsync(t->d_flags.p + n, 0, sizeof(uint32_t), s));
    r = scan_excl<uint32_t, uint32_t>(t, t->d_flags.p, t->d_pos.p, n + 1, t->scan32);
    if (r != VD_OK) return r;
    if (n) {
      k_range_compact<<<grid_blocks(t, n, 256), 256, 0, s>>>(t->d_sorted.p, n, t->d_flags.p, t->d_pos.p,
                                                             t->d_list[2].p);
      g_launches++;
      VD_CK(t, cudaGetLastError());
    }
    in_list = t->d_list[2].p;
    nin = (uint32_t)strided_count(range);
  }
  if (nin > 0) {
    r = clip_pass(t, 0, in_list, nin, t->d_list[0].p, t->d_list[1].p, extra);
    if (r != VD_OK) return r;
  }
  VD_CK(t, cudaEventRecord(t->ev[3], s));
  unsigned int novf = 0, ntab = 0;
  if (nin > 0) {
    r = read_ctl(t, &novf, &ntab);
    if (r != VD_OK) return r;
  }
  t->fallback[0] += novf;
  t->fallback[1] += ntab;
  // lists: [0] overflow, [1] table; [2] spare
  for (int guard = 0; guard < 64 && (novf > 0 || ntab > 0); ++guard) {
    if (ntab > 0) {
      if (t->order_complete) return fail(t, VD_ECUDA, "search order exhausted on a complete table");
      int k = std::max(1, t->order_k) * 2;
      r = upload_order(t, k);
      if (r != VD_OK) return r;
      // rerun table cells; overflows go to a fresh list, appended after novf
      std::swap(t->d_list[1], t->d_list[2]);
      r = clip_pass(t, 0, t->d_list[2].p, ntab, t->d_list[0].p + novf, t->d_list[1].p, extra);
      if (r != VD_OK) return r;
      unsigned int o2, t2;
      r = read_ctl(t, &o2, &t2);
      if (r != VD_OK) return r;
      t->fallback[1] += t2;
      t->fallback[0] += o2;
      novf += o2;
      ntab = t2;
      continue;
    }
    if (novf > 0) {
      // the slot layout's hand-offs to the full-rewrite first tier (48 faces,
      // every cell's layout equal in results), then medium capacity, then the
      // large and huge capacities for what remains
      unsigned int ntab_all = 0;
      // (for a few cells the extra pass's launch and read-back cost more than
      // the medium tier's slower per-cell build)
      const bool slots = t->fast_layout == VD_FAST_SLOTS && !(extra && extra->ex_verts) &&
                         novf >= (unsigned)kFullHandoffMin;
      for (int tier = slots ? -1 : 1; tier <= 3 && novf > 0;) {
        std::swap(t->d_list[0], t->d_list[2]);
        r = clip_pass(t, tier, t->d_list[2].p, novf, t->d_list[0].p, t->d_list[1].p + ntab_all, extra);
        if (r != VD_OK) return r;
        unsigned int o2, t2;
        r = read_ctl(t, &o2, &t2);
        if (r != VD_OK) return r;
        ntab_all += t2;
        if (tier == 3 && o2 > 0) return fail(t, VD_EOVERFLOW, "%u cells exceed the huge polytope capacity", o2);
        novf = o2;
        // few cells left after the medium tier: straight to the block tier,
        // which takes them all at once, so that a cell outgrowing the large
        // tier is not built twice
        int next = tier == -1 ? 1 : tier + 1;
        if (tier == 1 && novf > 0 && novf <= (unsigned)t->huge_direct_max) next = 3;
        tier = next;
      }
      novf = 0;
      ntab = ntab_all;
      t->fallback[1] += ntab_all;
    }
  }
  VD_CK(t, cudaEventRecord(t->ev[4], s));
  VD_CK(t, cudaMemcpyAsync(t->counters, t->d_counters.p, sizeof(t->counters), cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaStreamSynchronize(s));
  float a = 0, b = 0;
  cudaEventElapsedTime(&a, t->ev[2], t->ev[3]);
  cudaEventElapsedTime(&b, t->ev[3], t->ev[4]);
  t->timings[1] = a;
  t->timings[2] = b;
  t->timings[3] = t->timings[0] + a + b;
  return VD_OK;
}

int ensure_csr(vd_tess* t) {
  if (t->csr_valid) return VD_OK;
  const size_t n = t->ncells;
  cudaStream_t s = t->stream;
  VD_CK(t, t->d_nf64.ensure(n + 1, t->stream));
  VD_CK(t, t->d_csr_off.ensure(n + 1, t->stream));
  if (n) {
    k_nfaces_to_i64<<<grid_blocks(t, n, 256), 256, 0, s>>>(t->d_nf.p, n, t->d_nf64.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
  }
  VD_CK(t, cudaMemsetAsync(t->d_nf64.p + n, 0, sizeof(long long), s));
  int r = scan_excl<long long, long long>(t, t->d_nf64.p, t->d_csr_off.p, n + 1, t->scan64);
  if (r != VD_OK) return r;
  long long total = 0;
  VD_CK(t, cudaMemcpyAsync(&total, t->d_csr_off.p + n, sizeof(long long), cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaStreamSynchronize(s));
  t->csr_total = total;
  t->csr_valid = true;
  return VD_OK;
}

// bit k: wall k is curved (WallGeometry::is_planar false: every kind but
// planes and convex polyhedra)
uint32_t curved_bits(const vd_tess* t) {
  uint32_t m = 0;
  for (size_t k = 0; k < t->walls.size(); ++k)
    if (t->walls[k].kind != kWallPlane && t->walls[k].kind != kWallPolyhedron) m |= 1u << k;
  return m;
}

// bit k: the first wall with wall k's id is curved (walls.iter().find decides
// whether a face's id counts as a curved wall, tessellation.rs:250-256)
uint32_t first_curved_bits(const vd_tess* t) {
  const uint32_t c = curved_bits(t);
  uint32_t m = 0;
  for (size_t k = 0; k < t->walls.size(); ++k) {
    size_t f = 0;
    while (t->walls[f].id != t->walls[k].id) ++f;
    if ((c >> f) & 1u) m |= 1u << k;
  }
  return m;
}

// the ids of the cells whose mask is non-zero, in id order, into d_sel
int select_cells(vd_tess* t, const uint32_t* d_mask, uint32_t* nsel) {
  const size_t n = t->ngen;
  cudaStream_t s = t->stream;
  VD_CK(t, t->d_flags.ensure(n + 1, t->stream));
  VD_CK(t, t->d_pos.ensure(n + 1, t->stream));
  VD_CK(t, t->d_sel.ensure(n, t->stream));
  if (n) {
    k_nonzero_flags<<<grid_blocks(t, n, 256), 256, 0, s>>>(d_mask, n, t->d_flags.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
  }
  VD_CK(t, cudaMemsetAsync(t->d_flags.p + n, 0, sizeof(uint32_t), s));
  int r = scan_excl<uint32_t, uint32_t>(t, t->d_flags.p, t->d_pos.p, n + 1, t->scan32);
  if (r != VD_OK) return r;
  if (n) {
    k_compact_ids<<<grid_blocks(t, n, 256), 256, 0, s>>>(t->d_flags.p, t->d_pos.p, n, t->d_sel.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
  }
  uint32_t k = 0;
  VD_CK(t, cudaMemcpyAsync(&k, t->d_pos.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaStreamSynchronize(s));
  *nsel = k;
  return VD_OK;
}

// One seal or prune pass over the listed cells, with the fallbacks of
// run_calculate: a longer search order for cells that walk off a truncated
// one, the large-capacity kernel for polytopes that outgrow shared memory.
int seal_pass(vd_tess* t, const SealArgs& A, const uint32_t* items, uint32_t nitems,
              const WorkList* extra = nullptr) {
  cudaStream_t s = t->stream;
  if (nitems == 0) return VD_OK;
  // tier 0: shared memory, 1: large (global memory, a warp per cell), 2: huge (a block per cell)
  auto pass = [&](int tier, const uint32_t* list, uint32_t n, unsigned* novf, unsigned* ntab) -> int {
    VD_CK(t, cudaMemsetAsync(t->d_ctl.p, 0, 3 * sizeof(unsigned int), s));
    WorkList W;
    memset(&W, 0, sizeof(W));
    if (extra) W = *extra;
    W.items = list;
    W.nitems = n;
    W.cursor = t->d_ctl.p + kCtlCursor;
    W.ovf_list = t->d_list[0].p;
    W.ovf_count = t->d_ctl.p + kCtlOvfCount;
    W.tab_list = t->d_list[1].p;
    W.tab_count = t->d_ctl.p + kCtlTabCount;
    if (tier == 1) {
      int r = ensure_big(t, n);
      if (r == VD_OK) r = ensure_pool(t, n, faces_bound(t, kBigFaces, true));
      if (r != VD_OK) return r;
      VD_CK(t, launch_seal_big(make_desc(t), W, A, t->d_big.p, (int)t->big_warps, s));
    } else if (tier == 2) {
      int r = ensure_pool(t, n, faces_bound(t, kHugeFaces, true));
      if (r == VD_OK) r = ensure_huge(t, n);
      if (r != VD_OK) return r;
      VD_CK(t, launch_seal_block(make_desc(t), W, A, t->d_huge.p, (int)t->huge_blocks, s));
    } else {
      const ClipLaunchInfo& li = t->info64;
      const size_t want = (n + li.warps_per_block - 1) / li.warps_per_block;
      const int nblocks = (int)std::max<size_t>(1, std::min<size_t>(want, (size_t)t->num_sms * std::max(1, li.blocks_per_sm)));
      VD_CK(t, launch_seal_fast(make_desc(t), W, A, nblocks, s));
    }
    g_launches++;
    return read_ctl(t, novf, ntab);
  };
  // the input list lives in d_sel; overflow and table lists in d_list[0/1]
  unsigned novf = 0, ntab = 0;
  int r = pass(0, items, nitems, &novf, &ntab);
  for (int guard = 0; r == VD_OK && guard < 64 && (novf > 0 || ntab > 0); ++guard) {
    if (ntab > 0) {
      if (t->order_complete) return fail(t, VD_ECUDA, "search order exhausted on a complete table");
      r = upload_order(t, std::max(1, t->order_k) * 2);
      if (r != VD_OK) return r;
      // both lists are consumed before the pass refills them: move them aside
      VD_CK(t, cudaMemcpyAsync(t->d_list[2].p, t->d_list[1].p, ntab * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
      VD_CK(t, cudaMemcpyAsync(t->d_list[2].p + ntab, t->d_list[0].p, novf * sizeof(uint32_t),
                               cudaMemcpyDeviceToDevice, s));
      const unsigned n2 = ntab + novf;
      r = pass(0, t->d_list[2].p, n2, &novf, &ntab);
      continue;
    }
    VD_CK(t, cudaMemcpyAsync(t->d_list[2].p, t->d_list[0].p, novf * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    r = pass(1, t->d_list[2].p, novf, &novf, &ntab);
    // (cells that ran off the table as well are rerun from tier 0 with it, by
    // the loop, before any goes to the huge tier)
    if (r == VD_OK && novf > 0 && ntab == 0) {
      VD_CK(t, cudaMemcpyAsync(t->d_list[2].p, t->d_list[0].p, novf * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                               s));
      r = pass(2, t->d_list[2].p, novf, &novf, &ntab);
      if (r == VD_OK && novf > 0) return fail(t, VD_EOVERFLOW, "%u cells exceed the huge polytope capacity", novf);
    }
  }
  if (r == VD_OK && novf > 0) return fail(t, VD_EOVERFLOW, "%u cells exceed the polytope capacities", novf);
  return r;
}

// per-cell counts -> offsets (n + 1 entries, total at [n])
int count_offsets(vd_tess* t, DevBuf<int32_t>& cnt, DevBuf<long long>& off, size_t* total) {
  const size_t n = t->ngen;
  VD_CK(t, off.ensure(n + 1, t->stream));
  VD_CK(t, cudaMemsetAsync(cnt.p + n, 0, sizeof(int32_t), t->stream));
  int r = scan_excl<int32_t, long long>(t, cnt.p, off.p, n + 1, t->scan64);
  if (r != VD_OK) return r;
  long long tot = 0;
  VD_CK(t, cudaMemcpyAsync(&tot, off.p + n, sizeof(long long), cudaMemcpyDeviceToHost, t->stream));
  VD_CK(t, cudaStreamSynchronize(t->stream));
  *total = (size_t)tot;
  return VD_OK;
}

SealArgs seal_args(vd_tess* t, int mode) {
  SealArgs A;
  memset(&A, 0, sizeof(A));
  A.mode = mode;
  A.sealed = t->sealed ? 1 : 0;
  A.curved = curved_bits(t);
  A.fout = t->fout;
  A.s_nf = t->d_s_nf.p;
  A.s_fnb = t->d_s_fnb.p;
  A.s_pool_off = t->d_s_pool_off.p;
  A.s_pool_fnb = t->d_s_pool_fnb.p;
  A.s_mask = t->d_s_mask.p;
  A.c_nf = t->d_nf.p;
  A.c_fnb = t->d_fnb.p;
  A.c_pool_off = t->d_pool_off.p;
  A.c_pool_fnb = t->d_pool_fnb.p;
  A.c_mask = t->d_c_mask.p;
  A.seal_rec = t->d_seal_rec.p;
  A.prune_rec = t->d_prune_rec.p;
  A.prune_pos = t->d_prune_posrec.p;
  A.rec_cursor = t->d_rec_cursor.p;
  A.cnt = t->d_lcnt.p;
  A.pcnt = t->d_lpcnt.p;
  return A;
}

int check_ready(vd_tess* t) {
  if (!t) return VD_EINVAL;
  if (!t->calculated) return fail(t, VD_ESTATE, "no results: call vd_tess_calculate first");
  VD_CK(t, cudaSetDevice(t->device));
  return VD_OK;
}

}  // namespace

namespace vd {
void set_scratch_caps(vd_tess* t, size_t big_warps, size_t huge_blocks) {
  t->big_warps_cap = big_warps;
  t->huge_blocks_cap = huge_blocks;
}
}  // namespace vd

extern "C" {

const char* vd_last_error(const vd_tess* t) { return t ? t->err.c_str() : g_create_error.c_str(); }

int vd_tess_create(const double bmin[3], const double bmax[3], int nx, int ny, int nz, vd_tess** out) {
  if (!out || !bmin || !bmax) return fail(nullptr, VD_EINVAL, "null argument");
  *out = nullptr;
  if (nx <= 0 || ny <= 0 || nz <= 0 || nx > 16000 || ny > 16000 || nz > 16000)
    return fail(nullptr, VD_EINVAL, "grid resolution must be in [1, 16000]");
  if ((double)nx * ny * nz > 2.0e9) return fail(nullptr, VD_EINVAL, "too many bins");
  // A box without a positive, finite extent on every axis has no grid (the
  // reference's bin scale n / (max - min) would be infinite or NaN).
  for (int a = 0; a < 3; ++a)
    if (!(bmax[a] > bmin[a]) || !std::isfinite(bmin[a]) || !std::isfinite(bmax[a]) ||
        !std::isfinite(bmax[a] - bmin[a]))
      return fail(nullptr, VD_EINVAL, "bounding box axis %d: [%g, %g] has no positive finite extent", a, bmin[a],
                  bmax[a]);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(nullptr, VD_ECUDA, "no CUDA device: %s", cudaGetErrorString(e));
  vd_tess* t = new vd_tess();
  t->device = dev;
  cudaDeviceGetAttribute(&t->num_sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete t;
    return fail(nullptr, VD_ECUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
  }
  for (auto& ev : t->ev) cudaEventCreate(&ev);
  e = clip_fp64_info(&t->info64);
  if (e == cudaSuccess) e = clip_mixed_info(&t->infomx);
  for (int k = 0; k < 3 && e == cudaSuccess; ++k) {
    e = clip_sparse_info(false, 5 + k, &t->infosp64[k]);
    if (e == cudaSuccess) e = clip_sparse_info(true, 5 + k, &t->infospmx[k]);
  }
  if (e == cudaSuccess) e = clip_med_setup(&t->infomed);
  if (e == cudaSuccess) e = seal_setup();
  if (e != cudaSuccess) {
    const std::string m = cudaGetErrorString(e);
    vd_tess_destroy(t);
    return fail(nullptr, VD_ECUDA, "kernel setup: %s", m.c_str());
  }
  // Algorithm3DGrid::new (algo_3d_grid.rs:47-95)
  Grid& g = t->grid;
  const int n[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) {
    g.bmin[a] = bmin[a];
    g.bmax[a] = bmax[a];
    g.n[a] = n[a];
    g.scale[a] = (double)n[a] / (bmax[a] - bmin[a]);
    g.limit[a] = (double)n[a] - 1e-5;
    g.cs[a] = 1.0 / g.scale[a];
  }
  t->nbins = (size_t)nx * ny * nz;
  const double full = (2.0 * nx + 1) * (2.0 * ny + 1) * (2.0 * nz + 1);
  int r = upload_order(t, full <= (double)kCompleteOrderMax ? std::max(nx, std::max(ny, nz)) : 8);
  if (r == VD_OK) r = rebin(t);
  if (r != VD_OK) {
    g_create_error = t->err;
    vd_tess_destroy(t);
    return r;
  }
  *out = t;
  return VD_OK;
}

// A new bounding box and grid on an existing handle: device buffers are kept
// (they only grow), walls and generators are cleared.
int vd_tess_reset(vd_tess* t, const double bmin[3], const double bmax[3], int nx, int ny, int nz) {
  if (!t || !bmin || !bmax) return VD_EINVAL;
  if (nx <= 0 || ny <= 0 || nz <= 0 || nx > 16000 || ny > 16000 || nz > 16000)
    return fail(t, VD_EINVAL, "grid resolution must be in [1, 16000]");
  if ((double)nx * ny * nz > 2.0e9) return fail(t, VD_EINVAL, "too many bins");
  for (int a = 0; a < 3; ++a)
    if (!(bmax[a] > bmin[a]) || !std::isfinite(bmin[a]) || !std::isfinite(bmax[a]) ||
        !std::isfinite(bmax[a] - bmin[a]))
      return fail(t, VD_EINVAL, "bounding box axis %d: [%g, %g] has no positive finite extent", a, bmin[a],
                  bmax[a]);
  VD_CK(t, cudaSetDevice(t->device));
  Grid& g = t->grid;
  const int n[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) {
    g.bmin[a] = bmin[a];
    g.bmax[a] = bmax[a];
    g.n[a] = n[a];
    g.scale[a] = (double)n[a] / (bmax[a] - bmin[a]);
    g.limit[a] = (double)n[a] - 1e-5;
    g.cs[a] = 1.0 / g.scale[a];
  }
  t->nbins = (size_t)nx * ny * nz;
  t->walls.clear();
  t->planes.clear();
  t->ngen = 0;
  t->ncells = 0;
  t->calculated = false;
  t->csr_valid = false;
  const double full = (2.0 * nx + 1) * (2.0 * ny + 1) * (2.0 * nz + 1);
  int r = upload_order(t, full <= (double)kCompleteOrderMax ? std::max(nx, std::max(ny, nz)) : 8);
  if (r != VD_OK) return r;
  return rebin(t);
}

int vd_tess_destroy(vd_tess* t) {
  if (!t) return VD_OK;
  cudaSetDevice(t->device);
  if (t->stream) cudaStreamSynchronize(t->stream);
  t->d_order.release();
  t->d_planes.release();
  t->d_s_nf.release(); t->d_s_fnb.release(); t->d_s_pool_fnb.release(); t->d_s_pool_off.release();
  t->d_s_mask.release(); t->d_c_mask.release(); t->d_sel.release();
  t->d_seal_rec.release(); t->d_prune_rec.release(); t->d_prune_posrec.release(); t->d_rec_cursor.release();
  t->d_lcnt.release(); t->d_lpcnt.release(); t->d_loff.release(); t->d_lpoff.release();
  t->d_seal_log.release(); t->d_prune_log.release(); t->d_prune_pos.release();
  t->d_gen.release(); t->d_in.release(); t->d_tmp3.release();
  t->d_flags.release(); t->d_pos.release();
  t->d_bin_of.release(); t->d_bin_count.release(); t->d_bin_start.release(); t->d_cursor.release();
  t->d_ids.release(); t->d_ids_tmp.release(); t->d_big_list.release(); t->d_sorted.release();
  t->d_vol.release(); t->d_cen.release(); t->d_pool_area.release(); t->d_csr_area.release();
  t->d_nf.release(); t->d_nv.release(); t->d_fnb.release(); t->d_pool_fnb.release(); t->d_csr_ids.release();
  t->d_farea.release(); t->d_status.release(); t->d_pool_off.release(); t->d_csr_off.release();
  t->d_nf64.release(); t->d_ctl.release(); t->d_counters.release(); t->d_pool_cursor.release();
  for (auto& l : t->d_list) l.release();
  t->d_big.release();
  t->d_huge.release();
  for (auto& b : t->scan32) b.release();
  for (auto& b : t->scan64) b.release();
  t->d_ex_v.release(); t->d_ex_fc.release(); t->d_ex_fi.release(); t->d_ex_fn.release(); t->d_ex_sizes.release();
  t->d_bx_items.release(); t->d_bx_fc.release(); t->d_bx_fi.release(); t->d_bx_sizes.release();
  t->d_bx_fn.release(); t->d_bx_off.release(); t->d_bx_v.release();
  if (t->stream) cudaStreamSynchronize(t->stream);
  for (auto& ev : t->ev)
    if (ev) cudaEventDestroy(ev);
  if (t->stream) cudaStreamDestroy(t->stream);
  delete t;
  return VD_OK;
}

static int add_wall(vd_tess* t, const Wall& w, const double* planes = nullptr) {
  if (w.id > VD_WALL_ID_MAX) return fail(t, VD_EINVAL, "Wall ID must be <= %d", VD_WALL_ID_MAX);
  if ((int)t->walls.size() >= kMaxWalls) return fail(t, VD_EINVAL, "at most %d walls", kMaxWalls);
  VD_CK(t, cudaSetDevice(t->device));
  if (w.kind == kWallPolyhedron) {
    if ((int)(t->planes.size() / 6) + w.np > kMaxWallPlanes)
      return fail(t, VD_EINVAL, "at most %d polyhedron planes in all walls", kMaxWallPlanes);
    Wall wp = w;
    wp.p0 = (int)(t->planes.size() / 6);
    t->planes.insert(t->planes.end(), planes, planes + 6 * (size_t)w.np);
    VD_CK(t, t->d_planes.ensure(t->planes.size(), t->stream));
    VD_CK(t, cudaMemcpyAsync(t->d_planes.p, t->planes.data(), t->planes.size() * sizeof(double),
                             cudaMemcpyHostToDevice, t->stream));
    VD_CK(t, cudaStreamSynchronize(t->stream));
    t->walls.push_back(wp);
  } else {
    t->walls.push_back(w);
  }
  // prune_outside_generators (tessellation.rs:175-194)
  if (t->ngen == 0) return VD_OK;
  const size_t before = t->ngen;
  size_t kept = 0;
  int r = filter_into_gen(t, t->d_gen.p, before, &kept);
  if (r != VD_OK) return r;
  if (kept != before) return rebin(t);
  return VD_OK;
}

int vd_tess_add_wall_plane(vd_tess* t, const double point[3], const double normal[3], int id) {
  if (!t || !point || !normal) return VD_EINVAL;
  Wall w;
  memset(&w, 0, sizeof(w));
  w.kind = 0;
  w.id = id;
  for (int a = 0; a < 3; ++a) w.a[a] = point[a];
  // PlaneGeometry::new (wall_3d.rs:23-27)
  const double len = std::sqrt(normal[0] * normal[0] + normal[1] * normal[1] + normal[2] * normal[2]);
  if (len == 0.0) {
    w.n[0] = 0.0;
    w.n[1] = 0.0;
    w.n[2] = 1.0;
  } else {
    for (int a = 0; a < 3; ++a) w.n[a] = normal[a] / len;
  }
  return add_wall(t, w);
}

int vd_tess_add_wall_sphere(vd_tess* t, const double center[3], double radius, int id) {
  if (!t || !center) return VD_EINVAL;
  Wall w;
  memset(&w, 0, sizeof(w));
  w.kind = 1;
  w.id = id;
  w.r = radius;
  for (int a = 0; a < 3; ++a) w.a[a] = center[a];
  return add_wall(t, w);
}



int vd_tess_add_wall_cylinder(vd_tess* t, const double center[3], const double axis[3], double radius, int id) {
  if (!t || !center || !axis) return VD_EINVAL;
  Wall w;
  memset(&w, 0, sizeof(w));
  w.kind = kWallCylinder;
  w.id = id;
  w.r = radius;
  for (int a = 0; a < 3; ++a) w.a[a] = center[a];
  unit_axis(axis, w.n);
  return add_wall(t, w);
}

int vd_tess_add_wall_cone(vd_tess* t, const double tip[3], const double axis[3], double angle, int id) {
  if (!t || !tip || !axis) return VD_EINVAL;
  Wall w;
  memset(&w, 0, sizeof(w));
  w.kind = kWallCone;
  w.id = id;
  w.r = angle;
  // the reference evaluates angle.cos(), .sin(), .tan() with the host libm on
  // every call; they are evaluated here once, with the same libm
  w.ca = std::cos(angle);
  w.sa = std::sin(angle);
  w.ta = std::tan(angle);
  for (int a = 0; a < 3; ++a) w.a[a] = tip[a];
  unit_axis(axis, w.n);
  return add_wall(t, w);
}

int vd_tess_add_wall_torus(vd_tess* t, const double center[3], const double axis[3], double major_radius,
                           double minor_radius, int id) {
  if (!t || !center || !axis) return VD_EINVAL;
  Wall w;
  memset(&w, 0, sizeof(w));
  w.kind = kWallTorus;
  w.id = id;
  w.r = major_radius;
  w.r2 = minor_radius;
  for (int a = 0; a < 3; ++a) w.a[a] = center[a];
  unit_axis(axis, w.n);
  return add_wall(t, w);
}

int vd_tess_add_wall_polyhedron(vd_tess* t, const double* points, const double* normals, int nplanes, int id) {
  if (!t || nplanes < 0 || (nplanes > 0 && (!points || !normals))) return VD_EINVAL;
  Wall w;
  memset(&w, 0, sizeof(w));
  w.kind = kWallPolyhedron;
  w.id = id;
  w.np = nplanes;
  std::vector<double> pl(6 * (size_t)nplanes);
  for (int k = 0; k < nplanes; ++k)
    for (int a = 0; a < 3; ++a) {
      pl[6 * k + a] = points[3 * k + a];
      pl[6 * k + 3 + a] = normals[3 * k + a];
    }
  return add_wall(t, w, pl.data());
}

int vd_tess_clear_walls(vd_tess* t) {
  if (!t) return VD_EINVAL;
  t->walls.clear();
  t->planes.clear();
  return VD_OK;
}

static int set_generators_from_device(vd_tess* t, const double* d_src, size_t n, size_t* n_kept) {
  VD_CK(t, cudaEventRecord(t->ev[0], t->stream));
  int r = filter_into_gen(t, d_src, n, n_kept);
  if (r != VD_OK) return r;
  r = rebin(t);
  if (r != VD_OK) return r;
  VD_CK(t, cudaEventRecord(t->ev[1], t->stream));
  VD_CK(t, cudaEventSynchronize(t->ev[1]));
  cudaEventElapsedTime(&t->timings[0], t->ev[0], t->ev[1]);
  return VD_OK;
}

int vd_tess_set_generators(vd_tess* t, const double* xyz, size_t n, size_t* n_kept) {
  if (!t || (!xyz && n)) return VD_EINVAL;
  VD_CK(t, cudaSetDevice(t->device));
  if (n > 0xFFFFFFF0ull / 3) return fail(t, VD_EINVAL, "too many generators");
  // land the host copy in d_gen directly when no wall can drop rows
  DevBuf<double>& dst = t->walls.empty() ? t->d_gen : t->d_in;
  VD_CK(t, dst.ensure(3 * n, t->stream));
  if (n) VD_CK(t, cudaMemcpyAsync(dst.p, xyz, 3 * n * sizeof(double), cudaMemcpyHostToDevice, t->stream));
  return set_generators_from_device(t, dst.p, n, n_kept);
}

int vd_tess_set_generators_device(vd_tess* t, const double* d_xyz, size_t n, size_t* n_kept) {
  if (!t || (!d_xyz && n)) return VD_EINVAL;
  VD_CK(t, cudaSetDevice(t->device));
  if (n > 0xFFFFFFF0ull / 3) return fail(t, VD_EINVAL, "too many generators");
  // the filter reads d_xyz and writes d_gen, so the caller's buffer is never modified
  if (t->walls.empty()) {
    VD_CK(t, t->d_gen.ensure(3 * n, t->stream));
    if (n)
      VD_CK(t, cudaMemcpyAsync(t->d_gen.p, d_xyz, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, t->stream));
    return set_generators_from_device(t, t->d_gen.p, n, n_kept);
  }
  return set_generators_from_device(t, d_xyz, n, n_kept);
}

// Tessellation::random_generators (tessellation.rs:96-121) with an explicit
// seed: candidates in attempt order, batches of them generated and filtered
// on the device, the first `count` inside every wall kept, at most
// count * 1000 attempts.  Candidates are counter-based (splitmix64_at), so the
// batching does not change which points are kept.
int vd_tess_random_generators(vd_tess* t, size_t count, uint64_t seed, size_t* n_found) {
  if (!t) return VD_EINVAL;
  VD_CK(t, cudaSetDevice(t->device));
  if (count > 0xFFFFFFF0ull / 3) return fail(t, VD_EINVAL, "too many generators");
  cudaStream_t s = t->stream;
  const unsigned long long max_att = 1000ull * count;
  constexpr unsigned long long kMaxBatch = 1ull << 24;
  VD_CK(t, t->d_in.ensure(3 * count, s));
  const WallSet ws = wallset(t);
  size_t found = 0;
  unsigned long long att = 0;
  while (found < count && att < max_att) {
    const unsigned long long want = 2ull * (count - found) + 4096;
    const size_t B = (size_t)std::min(max_att - att, std::min(want, kMaxBatch));
    VD_CK(t, t->d_tmp3.ensure(3 * B, s));
    VD_CK(t, t->d_flags.ensure(B + 1, s));
    VD_CK(t, t->d_pos.ensure(B + 1, s));
    k_random_candidates<<<grid_blocks(t, B, 256), 256, 0, s>>>(seed, att, B, t->grid, ws, t->d_tmp3.p,
                                                               t->d_flags.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
    VD_CK(t, cudaMemsetAsync(t->d_flags.p + B, 0, sizeof(uint32_t), s));
    int r = scan_excl<uint32_t, uint32_t>(t, t->d_flags.p, t->d_pos.p, B + 1, t->scan32);
    if (r != VD_OK) return r;
    k_compact3_first<<<grid_blocks(t, B, 256), 256, 0, s>>>(t->d_tmp3.p, B, t->d_flags.p, t->d_pos.p,
                                                            (uint32_t)(count - found), t->d_in.p + 3 * found);
    g_launches++;
    VD_CK(t, cudaGetLastError());
    uint32_t acc = 0;
    VD_CK(t, cudaMemcpyAsync(&acc, t->d_pos.p + B, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    VD_CK(t, cudaStreamSynchronize(s));
    found += std::min<size_t>(acc, count - found);
    att += B;
  }
  size_t kept = 0;
  const int r = set_generators_from_device(t, t->d_in.p, found, &kept);
  if (r == VD_OK && n_found) *n_found = kept;
  return r;
}

// Wall::contains / Wall::cut and Algorithm3DGrid::get_bin_index on the host,
// with the functions the kernels use (wall_contains, wall_plane) and the
// binning's clamp-scale-truncate
int vd_wall_contains(const vd_wall_desc* d, const double point[3], int* inside) {
  if (!d || !point || !inside) return VD_EINVAL;
  Wall w;
  std::vector<double> planes;
  std::string err;
  if (!wall_from_desc(*d, &w, &planes, &err)) {
    set_thread_error(err.c_str());
    return VD_EINVAL;
  }
  *inside = wall_contains(w, planes.data(), point[0], point[1], point[2]) ? 1 : 0;
  return VD_OK;
}

int vd_wall_cut(const vd_wall_desc* d, const double generator[3], double* points, double* normals, int cap,
                int* n) {
  if (!d || !generator || !n || cap < 0 || (cap > 0 && (!points || !normals))) return VD_EINVAL;
  Wall w;
  std::vector<double> planes;
  std::string err;
  if (!wall_from_desc(*d, &w, &planes, &err)) {
    set_thread_error(err.c_str());
    return VD_EINVAL;
  }
  if (w.kind == kWallPolyhedron) {
    *n = w.np;
    for (int k = 0; k < w.np && k < cap; ++k)
      for (int a = 0; a < 3; ++a) {
        points[3 * k + a] = planes[6 * k + a];
        normals[3 * k + a] = planes[6 * k + 3 + a];
      }
    return VD_OK;
  }
  double p[3], q[3];
  *n = wall_plane(w, generator[0], generator[1], generator[2], p, q) ? 1 : 0;
  if (*n && cap > 0)
    for (int a = 0; a < 3; ++a) {
      points[a] = p[a];
      normals[a] = q[a];
    }
  return VD_OK;
}

int vd_search_order(const double bmin[3], const double bmax[3], int nx, int ny, int nz, int k, int32_t* dxyz,
                    double* min_d2, size_t cap, size_t* n, int* complete, double* bound) {
  if (!bmin || !bmax || !n || nx <= 0 || ny <= 0 || nz <= 0 || k <= 0 || (cap && (!dxyz || !min_d2)))
    return VD_EINVAL;
  Grid g;
  memset(&g, 0, sizeof(g));
  const int res[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) {
    g.bmin[a] = bmin[a];
    g.bmax[a] = bmax[a];
    g.n[a] = res[a];
    g.scale[a] = (double)res[a] / (bmax[a] - bmin[a]);
    g.limit[a] = (double)res[a] - 1e-5;
    g.cs[a] = 1.0 / g.scale[a];
  }
  std::vector<Offset> h;
  bool comp = false;
  double bd = 0.0;
  build_order(g, k, h, comp, bd);
  *n = h.size();
  if (complete) *complete = comp ? 1 : 0;
  if (bound) *bound = bd;
  for (size_t q = 0; q < h.size() && q < cap; ++q) {
    dxyz[3 * q] = h[q].dx;
    dxyz[3 * q + 1] = h[q].dy;
    dxyz[3 * q + 2] = h[q].dz;
    min_d2[q] = h[q].min_d2;
  }
  return VD_OK;
}

int vd_grid_bin_index(const double bmin[3], const double bmax[3], int nx, int ny, int nz, const double point[3],
                      size_t* index) {
  if (!bmin || !bmax || !point || !index || nx <= 0 || ny <= 0 || nz <= 0) return VD_EINVAL;
  const int n[3] = {nx, ny, nz};
  size_t idx = 0, stride = 1;
  for (int a = 0; a < 3; ++a) {
    const double scale = (double)n[a] / (bmax[a] - bmin[a]);
    const double limit = (double)n[a] - 1e-5;
    double u = (point[a] - bmin[a]) * scale;
    if (u < 0.0) u = 0.0;
    if (u > limit) u = limit;
    idx += (u > 0.0 ? (size_t)u : 0) * stride;
    stride *= (size_t)n[a];
  }
  *index = idx;
  return VD_OK;
}

// Tessellation::read_generators / import_generators (tessellation.rs:126-171):
// parsed on the host, then the set_generators path
int vd_tess_read_generators(vd_tess* t, const char* text, size_t len, size_t* n_kept) {
  if (!t || (!text && len)) return VD_EINVAL;
  std::vector<double> xyz;
  std::string err;
  if (!parse_generators(text, len, &xyz, &err)) return fail(t, VD_EINVAL, "%s", err.c_str());
  return vd_tess_set_generators(t, xyz.data(), xyz.size() / 3, n_kept);
}

int vd_tess_import_generators(vd_tess* t, const char* path, size_t* n_kept) {
  if (!t || !path) return VD_EINVAL;
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(t, VD_EIO, "cannot open %s", path);
  std::string text;
  char buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, got);
  const bool bad = std::ferror(f) != 0;
  std::fclose(f);
  if (bad) return fail(t, VD_EIO, "cannot read %s", path);
  return vd_tess_read_generators(t, text.data(), text.size(), n_kept);
}

// Tessellation::set_generator + Algorithm3DGrid::update_generator
// (tessellation.rs:71-92, algo_3d_grid.rs:132-143).  The bin change uses the
// reference's swap_remove/push, so in-bin order follows the reference's.
int vd_tess_set_generator(vd_tess* t, size_t index, const double xyz[3]) {
  if (!t || !xyz) return VD_EINVAL;
  VD_CK(t, cudaSetDevice(t->device));
  if (index >= t->ngen) return VD_OK;
  for (const Wall& w : t->walls)
    if (!wall_contains(w, t->planes.data(), xyz[0], xyz[1], xyz[2])) return VD_OK;
  cudaStream_t s = t->stream;
  const size_t n = t->ngen, nb = t->nbins;
  std::vector<uint32_t> start(nb + 1), ids(n), bin_of(n);
  VD_CK(t, cudaMemcpyAsync(start.data(), t->d_bin_start.p, (nb + 1) * 4, cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaMemcpyAsync(ids.data(), t->d_ids.p, n * 4, cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaMemcpyAsync(bin_of.data(), t->d_bin_of.p, n * 4, cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaStreamSynchronize(s));
  const Grid& g = t->grid;
  auto axis = [](double v, double lo, double sc, double lim) -> uint32_t {
    double u = (v - lo) * sc;
    if (u < 0.0) u = 0.0;
    if (u > lim) u = lim;
    return u > 0.0 ? (uint32_t)u : 0u;
  };
  const uint32_t nbin = axis(xyz[0], g.bmin[0], g.scale[0], g.limit[0]) +
                        axis(xyz[1], g.bmin[1], g.scale[1], g.limit[1]) * (uint32_t)g.n[0] +
                        axis(xyz[2], g.bmin[2], g.scale[2], g.limit[2]) * (uint32_t)g.n[0] * (uint32_t)g.n[1];
  const uint32_t obin = bin_of[index];
  if (nbin != obin) {
    std::vector<std::vector<uint32_t>> bins(nb);
    for (size_t b = 0; b < nb; ++b) bins[b].assign(ids.begin() + start[b], ids.begin() + start[b + 1]);
    auto& ob = bins[obin];
    for (size_t k = 0; k < ob.size(); ++k)
      if (ob[k] == index) {
        ob[k] = ob.back();  // swap_remove
        ob.pop_back();
        break;
      }
    bins[nbin].push_back((uint32_t)index);
    bin_of[index] = nbin;
    size_t o = 0;
    for (size_t b = 0; b < nb; ++b) {
      start[b] = (uint32_t)o;
      for (uint32_t v : bins[b]) ids[o++] = v;
    }
    start[nb] = (uint32_t)o;
    VD_CK(t, cudaMemcpyAsync(t->d_bin_start.p, start.data(), (nb + 1) * 4, cudaMemcpyHostToDevice, s));
    VD_CK(t, cudaMemcpyAsync(t->d_ids.p, ids.data(), n * 4, cudaMemcpyHostToDevice, s));
    VD_CK(t, cudaMemcpyAsync(t->d_bin_of.p, bin_of.data(), n * 4, cudaMemcpyHostToDevice, s));
  }
  VD_CK(t, cudaMemcpyAsync(t->d_gen.p + 3 * index, xyz, 3 * sizeof(double), cudaMemcpyHostToDevice, s));
  k_gather_sorted<<<grid_blocks(t, n, 256), 256, 0, s>>>(t->d_ids.p, t->d_gen.p, n, t->d_sorted.p);
  g_launches++;
  VD_CK(t, cudaGetLastError());
  int ro = build_occupancy(t);
  if (ro != VD_OK) return ro;
  VD_CK(t, cudaStreamSynchronize(s));
  t->calculated = false;
  t->csr_valid = false;
  return VD_OK;
}

int vd_tess_count_generators(const vd_tess* t, size_t* n) {
  if (!t || !n) return VD_EINVAL;
  *n = t->ngen;
  return VD_OK;
}

int vd_tess_get_generators(vd_tess* t, double* xyz) {
  if (!t || (!xyz && t->ngen)) return VD_EINVAL;
  VD_CK(t, cudaSetDevice(t->device));
  if (t->ngen)
    VD_CK(t, cudaMemcpyAsync(xyz, t->d_gen.p, 3 * t->ngen * sizeof(double), cudaMemcpyDeviceToHost, t->stream));
  VD_CK(t, cudaStreamSynchronize(t->stream));
  return VD_OK;
}

int vd_tess_set_precision(vd_tess* t, int precision) {
  if (!t) return VD_EINVAL;
  if (precision != VD_PREC_FP64 && precision != VD_PREC_MIXED) return fail(t, VD_EINVAL, "unknown precision");
  t->precision = precision;
  return VD_OK;
}

int vd_debug_fail_allocations(int count) {
  g_fail_allocs.store(count > 0 ? count : 0);
  return VD_OK;
}

int vd_tess_set_fast_layout(vd_tess* t, int layout) {
  if (!t) return VD_EINVAL;
  if (layout != VD_FAST_SLOTS && layout != VD_FAST_FULL) return fail(t, VD_EINVAL, "unknown fast-tier layout");
  t->fast_layout = layout;
  return VD_OK;
}

int vd_tess_set_tuning(vd_tess* t, const vd_tuning* k) {
  if (!t || !k) return VD_EINVAL;
  if (k->fast_layout != 0 && k->fast_layout != VD_FAST_FULL)
    return fail(t, VD_EINVAL, "unknown fast-tier layout %d", k->fast_layout);
  if (k->fast_blocks_per_sm != 0 && (k->fast_blocks_per_sm < 5 || k->fast_blocks_per_sm > 7))
    return fail(t, VD_EINVAL, "fast_blocks_per_sm must be 5, 6 or 7");
  if (k->huge_direct_max < 0 || k->huge_blocks_max < 0 || k->huge_blocks_max > 256 || k->huge_narrow_max < 0)
    return fail(t, VD_EINVAL, "huge-tier settings out of range");
  t->fast_layout = k->fast_layout;
  t->fast_minb = k->fast_blocks_per_sm;
  t->huge_direct_max = k->huge_direct_max ? k->huge_direct_max : 64;
  t->huge_blocks_max = k->huge_blocks_max ? k->huge_blocks_max : kHugeBlocksMax;
  t->huge_narrow_max = k->huge_narrow_max ? k->huge_narrow_max : kHugeNarrowDefault;
  t->noop_run = k->noop_run ? k->noop_run : kNoopRunDefault;
  return VD_OK;
}

int vd_tess_get_tuning(const vd_tess* t, vd_tuning* k) {
  if (!t || !k) return VD_EINVAL;
  k->fast_layout = t->fast_layout;
  k->fast_blocks_per_sm = fast_minb_for(t);
  k->huge_direct_max = t->huge_direct_max;
  k->huge_blocks_max = t->huge_blocks_max;
  k->huge_narrow_max = t->huge_narrow_max;
  k->noop_run = t->noop_run;
  return VD_OK;
}

int vd_tess_set_instrumentation(vd_tess* t, int on) {
  if (!t) return VD_EINVAL;
  t->instrument = on != 0;
  return VD_OK;
}

int vd_tess_calculate(vd_tess* t) {
  if (!t) return VD_EINVAL;
  VD_CK(t, cudaSetDevice(t->device));
  t->calculated = false;
  t->csr_valid = false;
  t->sealed = false;
  t->nseal = t->nprune = t->nprune_pos = 0;
  int r = run_calculate(t);
  if (r != VD_OK) return r;
  t->ncells = t->ngen;
  t->range_begin = 0;
  t->range_end = t->ngen;
  t->range_chunk = 1;
  t->range_stride = 1;
  t->range_phase = 0;
  t->calculated = true;
  return VD_OK;
}

int vd_tess_calculate_strided(vd_tess* t, size_t begin, size_t end, size_t chunk, size_t stride, size_t phase) {
  if (!t) return VD_EINVAL;
  if (begin > end || end > t->ngen)
    return fail(t, VD_EINVAL, "cell range [%zu, %zu) is not inside [0, %zu)", begin, end, t->ngen);
  if (chunk == 0 || stride == 0 || phase >= stride)
    return fail(t, VD_EINVAL, "chunk %zu, stride %zu, phase %zu: need chunk >= 1 and phase < stride", chunk,
                stride, phase);
  VD_CK(t, cudaSetDevice(t->device));
  t->calculated = false;
  t->csr_valid = false;
  const size_t range[5] = {begin, end, chunk, stride, phase};
  t->sealed = false;
  t->nseal = t->nprune = t->nprune_pos = 0;
  int r = run_calculate(t, nullptr, nullptr, range);
  if (r != VD_OK) return r;
  t->ncells = t->ngen;
  t->range_begin = begin;
  t->range_end = end;
  t->range_chunk = chunk;
  t->range_stride = stride;
  t->range_phase = phase;
  t->calculated = true;
  return VD_OK;
}

int vd_tess_calculate_range(vd_tess* t, size_t begin, size_t end) {
  return vd_tess_calculate_strided(t, begin, end, 1, 1, 0);
}

int vd_tess_calculate_sealed(vd_tess* t) {
  int r = vd_tess_calculate(t);
  if (r != VD_OK) return r;
  const size_t n = t->ngen;
  cudaStream_t s = t->stream;
  // the topology before any cell changes (tessellation.rs:242-261)
  unsigned long long pool_used = 0;
  VD_CK(t, cudaMemcpyAsync(&pool_used, t->d_pool_cursor.p, sizeof(pool_used), cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaStreamSynchronize(s));
  VD_CK(t, t->d_s_nf.ensure(n, t->stream));
  VD_CK(t, t->d_s_fnb.ensure(n * (size_t)t->fout, t->stream));
  VD_CK(t, t->d_s_pool_off.ensure(n, t->stream));
  VD_CK(t, t->d_s_pool_fnb.ensure(std::max<unsigned long long>(pool_used, 1), t->stream));
  VD_CK(t, t->d_s_mask.ensure(n, t->stream));
  if (n) {
    VD_CK(t, cudaMemcpyAsync(t->d_s_nf.p, t->d_nf.p, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    VD_CK(t, cudaMemcpyAsync(t->d_s_fnb.p, t->d_fnb.p, n * (size_t)t->fout * sizeof(int32_t),
                             cudaMemcpyDeviceToDevice, s));
    VD_CK(t, cudaMemcpyAsync(t->d_s_pool_off.p, t->d_pool_off.p, n * sizeof(long long), cudaMemcpyDeviceToDevice, s));
    if (pool_used)
      VD_CK(t, cudaMemcpyAsync(t->d_s_pool_fnb.p, t->d_pool_fnb.p, pool_used * sizeof(int32_t),
                               cudaMemcpyDeviceToDevice, s));
  }
  VD_CK(t, launch_curved_mask(t->d_s_nf.p, t->d_s_fnb.p, t->d_s_pool_off.p, t->d_s_pool_fnb.p, t->fout,
                              (uint32_t)n, make_desc(t), first_curved_bits(t), t->d_s_mask.p,
                              grid_blocks(t, n, 256), s));
  g_launches++;
  uint32_t nsel = 0;
  r = select_cells(t, t->d_s_mask.p, &nsel);
  if (r != VD_OK) return r;
  // logs: at most one entry per (face, curved wall) of a selected cell;
  // entries of an attempt that a larger pass redoes repeat (up to three
  // attempts: shared memory, large, huge), so three times that
  const uint32_t cap = (uint32_t)std::min<size_t>((size_t)3 * nsel * t->fout * (size_t)std::max<int>(1, __builtin_popcount(curved_bits(t))) + 1024, 1u << 30);
  VD_CK(t, t->d_seal_rec.ensure(cap, t->stream));
  VD_CK(t, t->d_rec_cursor.ensure(2, t->stream));
  VD_CK(t, t->d_lcnt.ensure(n + 1, t->stream));
  VD_CK(t, cudaMemsetAsync(t->d_rec_cursor.p, 0, 2 * sizeof(unsigned int), s));
  VD_CK(t, cudaMemsetAsync(t->d_lcnt.p, 0, (n + 1) * sizeof(int32_t), s));
  SealArgs A = seal_args(t, 1);
  A.rec_cap = cap;
  r = seal_pass(t, A, t->d_sel.p, nsel);
  if (r != VD_OK) return r;
  unsigned int used[2];
  VD_CK(t, cudaMemcpyAsync(used, t->d_rec_cursor.p, sizeof(used), cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaStreamSynchronize(s));
  if (used[0] > cap) return fail(t, VD_ENOMEM, "seal log exceeds its buffer (%u records)", used[0]);
  size_t total = 0;
  r = count_offsets(t, t->d_lcnt, t->d_loff, &total);
  if (r != VD_OK) return r;
  VD_CK(t, t->d_seal_log.ensure(3 * total, t->stream));
  VD_CK(t, launch_seal_log_place(t->d_seal_rec.p, used[0], t->d_loff.p, t->d_seal_log.p,
                                 grid_blocks(t, used[0], 256), s));
  g_launches++;
  VD_CK(t, cudaStreamSynchronize(s));
  t->nseal = total;
  t->sealed = true;
  t->csr_valid = false;
  return VD_OK;
}

int vd_tess_prune_boundaries(vd_tess* t) {
  int r = check_ready(t);
  if (r != VD_OK) return r;
  const size_t n = t->ngen;
  cudaStream_t s = t->stream;
  VD_CK(t, t->d_c_mask.ensure(n, t->stream));
  VD_CK(t, launch_curved_mask(t->d_nf.p, t->d_fnb.p, t->d_pool_off.p, t->d_pool_fnb.p, t->fout, (uint32_t)n,
                              make_desc(t), first_curved_bits(t), t->d_c_mask.p, grid_blocks(t, n, 256), s));
  g_launches++;
  uint32_t nsel = 0;
  r = select_cells(t, t->d_c_mask.p, &nsel);
  if (r != VD_OK) return r;
  const size_t per = (size_t)t->fout * (size_t)std::max<int>(1, __builtin_popcount(curved_bits(t)));
  const uint32_t cap = (uint32_t)std::min<size_t>((size_t)nsel * per + 1024, 1u << 30);
  const uint32_t pcap = (uint32_t)std::min<size_t>((size_t)nsel * per * 8 + 4096, 1u << 30);
  VD_CK(t, t->d_prune_rec.ensure(cap, t->stream));
  VD_CK(t, t->d_prune_posrec.ensure(pcap, t->stream));
  VD_CK(t, t->d_rec_cursor.ensure(2, t->stream));
  VD_CK(t, t->d_lcnt.ensure(n + 1, t->stream));
  VD_CK(t, t->d_lpcnt.ensure(n + 1, t->stream));
  VD_CK(t, cudaMemsetAsync(t->d_rec_cursor.p, 0, 2 * sizeof(unsigned int), s));
  VD_CK(t, cudaMemsetAsync(t->d_lcnt.p, 0, (n + 1) * sizeof(int32_t), s));
  VD_CK(t, cudaMemsetAsync(t->d_lpcnt.p, 0, (n + 1) * sizeof(int32_t), s));
  SealArgs A = seal_args(t, 2);
  A.rec_cap = cap;
  A.pos_cap = pcap;
  r = seal_pass(t, A, t->d_sel.p, nsel);
  if (r != VD_OK) return r;
  unsigned int used[2];
  VD_CK(t, cudaMemcpyAsync(used, t->d_rec_cursor.p, sizeof(used), cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaStreamSynchronize(s));
  if (used[0] > cap || used[1] > pcap) return fail(t, VD_ENOMEM, "prune log exceeds its buffer");
  size_t total = 0, ptotal = 0;
  r = count_offsets(t, t->d_lcnt, t->d_loff, &total);
  if (r != VD_OK) return r;
  r = count_offsets(t, t->d_lpcnt, t->d_lpoff, &ptotal);
  if (r != VD_OK) return r;
  VD_CK(t, t->d_prune_log.ensure(4 * total, t->stream));
  VD_CK(t, t->d_prune_pos.ensure(3 * ptotal, t->stream));
  VD_CK(t, launch_prune_log_place(t->d_prune_rec.p, used[0], t->d_prune_posrec.p, used[1], t->d_loff.p,
                                  t->d_lpoff.p, t->d_prune_log.p, t->d_prune_pos.p,
                                  grid_blocks(t, std::max(used[0], used[1]), 256), s));
  g_launches++;
  VD_CK(t, cudaStreamSynchronize(s));
  t->nprune = total;
  t->nprune_pos = ptotal;
  return VD_OK;
}

int vd_tess_seal_log(vd_tess* t, int32_t* out, size_t* n) {
  if (!t || !n) return VD_EINVAL;
  *n = 3 * t->nseal;
  if (out && t->nseal) {
    VD_CK(t, cudaMemcpyAsync(out, t->d_seal_log.p, 3 * t->nseal * sizeof(int32_t), cudaMemcpyDeviceToHost, t->stream));
    VD_CK(t, cudaStreamSynchronize(t->stream));
  }
  return VD_OK;
}

int vd_tess_prune_log(vd_tess* t, int32_t* entries, size_t* n_entries, double* positions, size_t* n_positions) {
  if (!t || !n_entries || !n_positions) return VD_EINVAL;
  *n_entries = 4 * t->nprune;
  *n_positions = 3 * t->nprune_pos;
  if (entries && t->nprune)
    VD_CK(t, cudaMemcpyAsync(entries, t->d_prune_log.p, 4 * t->nprune * sizeof(int32_t), cudaMemcpyDeviceToHost,
                             t->stream));
  if (positions && t->nprune_pos)
    VD_CK(t, cudaMemcpyAsync(positions, t->d_prune_pos.p, 3 * t->nprune_pos * sizeof(double),
                             cudaMemcpyDeviceToHost, t->stream));
  VD_CK(t, cudaStreamSynchronize(t->stream));
  return VD_OK;
}

int vd_tess_relax(vd_tess* t) {
  int r = check_ready(t);
  if (r != VD_OK) return r;
  const size_t n = std::min(t->ncells, t->ngen);
  VD_CK(t, t->d_in.ensure(3 * n, t->stream));
  if (n) {
    k_relax<<<grid_blocks(t, n, 256), 256, 0, t->stream>>>(t->d_gen.p, t->d_nv.p, t->d_cen.p, n, t->d_in.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
  }
  // Tessellation::set_generators on the new positions (re-filter, re-bin)
  if (t->walls.empty()) {
    std::swap(t->d_gen, t->d_in);
    r = set_generators_from_device(t, t->d_gen.p, n, nullptr);
  } else {
    r = set_generators_from_device(t, t->d_in.p, n, nullptr);
  }
  return r;
}

int vd_tess_count_cells(const vd_tess* t, size_t* n) {
  if (!t || !n) return VD_EINVAL;
  *n = t->calculated ? t->ncells : 0;
  return VD_OK;
}

int vd_tess_get_cell_summaries(vd_tess* t, double* volume, double* centroid3, int32_t* n_faces) {
  int r = check_ready(t);
  if (r != VD_OK) return r;
  const size_t n = t->ncells;
  cudaStream_t s = t->stream;
  if (n) {
    if (volume) VD_CK(t, cudaMemcpyAsync(volume, t->d_vol.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (centroid3)
      VD_CK(t, cudaMemcpyAsync(centroid3, t->d_cen.p, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (n_faces) VD_CK(t, cudaMemcpyAsync(n_faces, t->d_nf.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  }
  VD_CK(t, cudaStreamSynchronize(s));
  return VD_OK;
}

int vd_tess_total_faces(vd_tess* t, int64_t* total) {
  int r = check_ready(t);
  if (r != VD_OK) return r;
  if (!total) return VD_EINVAL;
  r = ensure_csr(t);
  if (r != VD_OK) return r;
  *total = t->csr_total;
  return VD_OK;
}

static int get_csr(vd_tess* t, int64_t* offsets, int32_t* ids, double* areas) {
  int r = check_ready(t);
  if (r != VD_OK) return r;
  r = ensure_csr(t);
  if (r != VD_OK) return r;
  const size_t n = t->ncells;
  cudaStream_t s = t->stream;
  const size_t tot = (size_t)t->csr_total;
  if (ids) VD_CK(t, t->d_csr_ids.ensure(tot, t->stream));
  if (areas) VD_CK(t, t->d_csr_area.ensure(tot, t->stream));
  if (n && tot) {
    const int blocks = grid_blocks(t, n * 32, 256);
    k_csr_gather<<<blocks, 256, 0, s>>>(t->d_nf.p, n, t->d_csr_off.p, t->fout, t->d_fnb.p, t->d_farea.p,
                                        t->d_pool_fnb.p, t->d_pool_area.p, t->d_pool_off.p,
                                        ids ? t->d_csr_ids.p : nullptr, areas ? t->d_csr_area.p : nullptr);
    g_launches++;
    VD_CK(t, cudaGetLastError());
    if (ids) VD_CK(t, cudaMemcpyAsync(ids, t->d_csr_ids.p, tot * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    if (areas) VD_CK(t, cudaMemcpyAsync(areas, t->d_csr_area.p, tot * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  if (offsets)
    VD_CK(t, cudaMemcpyAsync(offsets, t->d_csr_off.p, (n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaStreamSynchronize(s));
  return VD_OK;
}

int vd_tess_get_neighbors(vd_tess* t, int64_t* offsets, int32_t* ids) {
  if (!ids) return VD_EINVAL;
  return get_csr(t, offsets, ids, nullptr);
}

int vd_tess_get_face_areas(vd_tess* t, int64_t* offsets, double* areas) {
  if (!areas) return VD_EINVAL;
  return get_csr(t, offsets, nullptr, areas);
}

// Recomputes cell i alone with polytope export.  The computation is
// deterministic, so the polytope is the one calculate() built.
int vd_tess_get_cell(vd_tess* t, size_t i, int32_t* n_vertices, int32_t* n_faces, int32_t* n_face_indices,
                     double* vertices, uint32_t* face_counts, uint32_t* face_indices, int32_t* face_neighbors) {
  int r = check_ready(t);
  if (r != VD_OK) return r;
  if (i >= t->ncells) return fail(t, VD_EINVAL, "cell index %zu out of range", i);
  if (!cell_computed(t, i)) {
    // outside the range of the last calculate_range: an empty cell
    if (n_vertices) *n_vertices = 0;
    if (n_faces) *n_faces = 0;
    if (n_face_indices) *n_face_indices = 0;
    return VD_OK;
  }
  cudaStream_t s = t->stream;
  const int cv = 65534, cf = 32767, ch = 196608;  // the huge tier's capacities
  VD_CK(t, t->d_ex_v.ensure(3 * cv, t->stream));
  VD_CK(t, t->d_ex_fc.ensure(cf, t->stream));
  VD_CK(t, t->d_ex_fi.ensure(ch, t->stream));
  VD_CK(t, t->d_ex_fn.ensure(cf, t->stream));
  VD_CK(t, t->d_ex_sizes.ensure(4, t->stream));
  VD_CK(t, cudaMemsetAsync(t->d_ex_sizes.p, 0, 4 * sizeof(int32_t), s));
  WorkList ex;
  memset(&ex, 0, sizeof(ex));
  ex.ex_verts = t->d_ex_v.p;
  ex.ex_fc = t->d_ex_fc.p;
  ex.ex_fi = t->d_ex_fi.p;
  ex.ex_fn = t->d_ex_fn.p;
  ex.ex_sizes = t->d_ex_sizes.p;
  ex.ex_cap_v = cv;
  ex.ex_cap_f = cf;
  ex.ex_cap_h = ch;
  // keep the calculate() counters and timings of the full run
  unsigned long long saved[kNumCounters];
  memcpy(saved, t->counters, sizeof(saved));
  float st[4];
  memcpy(st, t->timings, sizeof(st));
  unsigned long long sf[2] = {t->fallback[0], t->fallback[1]};
  const uint32_t cell = (uint32_t)i;
  if (t->sealed) {
    // the sealed polytope: rebuilt with the seal clips, nothing logged
    VD_CK(t, t->d_sel.ensure(std::max<size_t>(t->ngen, 1), t->stream));
    VD_CK(t, cudaMemcpyAsync(t->d_sel.p, &cell, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    SealArgs A = seal_args(t, 1);
    A.cnt = nullptr;
    A.rec_cap = 0;
    r = seal_pass(t, A, t->d_sel.p, 1, &ex);
  } else {
    r = run_calculate(t, &ex, &cell);
  }
  memcpy(t->counters, saved, sizeof(saved));
  memcpy(t->timings, st, sizeof(st));
  t->fallback[0] = sf[0];
  t->fallback[1] = sf[1];
  if (r != VD_OK) return r;
  int32_t sz[4];
  VD_CK(t, cudaMemcpyAsync(sz, t->d_ex_sizes.p, sizeof(sz), cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaStreamSynchronize(s));
  if (n_vertices) *n_vertices = sz[0];
  if (n_faces) *n_faces = sz[1];
  if (n_face_indices) *n_face_indices = sz[2];
  if (vertices && sz[0])
    VD_CK(t, cudaMemcpyAsync(vertices, t->d_ex_v.p, 3 * (size_t)sz[0] * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (face_counts && sz[1])
    VD_CK(t, cudaMemcpyAsync(face_counts, t->d_ex_fc.p, (size_t)sz[1] * 4, cudaMemcpyDeviceToHost, s));
  if (face_neighbors && sz[1])
    VD_CK(t, cudaMemcpyAsync(face_neighbors, t->d_ex_fn.p, (size_t)sz[1] * 4, cudaMemcpyDeviceToHost, s));
  if (face_indices && sz[2])
    VD_CK(t, cudaMemcpyAsync(face_indices, t->d_ex_fi.p, (size_t)sz[2] * 4, cudaMemcpyDeviceToHost, s));
  VD_CK(t, cudaStreamSynchronize(s));
  return VD_OK;
}

// Tessellation::cells / map (tessellation.rs:391-412, 524-526) for the cells
// [begin, end): sizes, offsets and, when the arrays are given, every polytope.
// The device passes rebuild the cells with calculate()'s code (and the seal
// clips, when the tessellation is sealed): first with the shared-memory
// capacities, then the cells that overflowed with the medium ones, then with
// the large ones in global scratch; the few cells beyond those go through
// get_cell.
int vd_tess_export_cells(vd_tess* t, size_t begin, size_t end, int64_t* v_off, int64_t* f_off, int64_t* h_off,
                         double* vertices, uint32_t* face_counts, uint32_t* face_indices, int32_t* face_neighbors) {
  int r = check_ready(t);
  if (r != VD_OK) return r;
  if (!v_off || !f_off || !h_off) return VD_EINVAL;
  if (begin > end || end > t->ncells) return fail(t, VD_EINVAL, "bad cell range [%zu, %zu)", begin, end);
  const bool fill = vertices || face_counts || face_indices || face_neighbors;
  if (fill && !(vertices && face_counts && face_indices && face_neighbors))
    return fail(t, VD_EINVAL, "give all four polytope arrays, or none for the sizes");
  if (end - begin > 0xFFFFFFF0ull) return fail(t, VD_EINVAL, "range too large");
  if (t->range_stride > 1)
    return fail(t, VD_ESTATE, "the last calculate computed interleaved chunks of cells; export after a "
                              "calculate or calculate_range");
  cudaStream_t s = t->stream;
  const size_t n = end - begin;
  // only the cells of the last calculate's range have polytopes
  const size_t lo = std::max(begin, t->range_begin), hi = std::min(end, t->range_end);
  std::vector<int32_t> sz(3 * n, 0);
  std::vector<size_t> host_cells;
  const bool device = hi > lo;
  ExportArgs A;
  memset(&A, 0, sizeof(A));
  TessDesc T = make_desc(t);
  // a sealed tessellation's seal clips, as get_cell applies them: nothing logged
  SealArgs SA = seal_args(t, 1);
  SA.cnt = nullptr;
  SA.rec_cap = 0;
  // the item list of each tier inside d_bx_items: all cells of the range (in
  // the spatial order), then the medium tier's, then the large tier's
  const size_t nr = hi - lo;
  size_t tier_at[3] = {0, nr, nr};
  uint32_t tier_n[3] = {(uint32_t)nr, 0, 0};
  auto run_tier = [&](int pass, int tier) -> int {
    if (tier == 2) {
      int rb = ensure_big(t, tier_n[2]);
      if (rb != VD_OK) return rb;
    }
    VD_CK(t, cudaMemsetAsync(t->d_ctl.p, 0, 3 * sizeof(unsigned int), s));
    A.items = t->d_bx_items.p + tier_at[tier];
    A.nitems = tier_n[tier];
    void* scratch = tier == 2 ? (void*)t->d_big.p : nullptr;
    const int nwarps = tier == 2 ? (int)t->big_warps : 0;
    VD_CK(t, t->sealed ? launch_seal_export_cells(T, A, SA, pass, tier, t->num_sms, scratch, nwarps, s)
                       : launch_export_cells(T, A, pass, tier, t->num_sms, scratch, nwarps, s));
    g_launches++;
    return VD_OK;
  };
  if (device) {
    const size_t all = t->ncells;
    VD_CK(t, t->d_flags.ensure(all + 1, s));
    VD_CK(t, t->d_pos.ensure(all + 1, s));
    VD_CK(t, t->d_bx_items.ensure(3 * nr, s));
    VD_CK(t, t->d_bx_sizes.ensure(3 * n, s));
    k_range_flags<<<grid_blocks(t, all, 256), 256, 0, s>>>(t->d_sorted.p, all, (long long)lo, (long long)hi, 1LL,
                                                         1LL, 0LL, t->d_flags.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
    VD_CK(t, cudaMemsetAsync(t->d_flags.p + all, 0, sizeof(uint32_t), s));
    r = scan_excl<uint32_t, uint32_t>(t, t->d_flags.p, t->d_pos.p, all + 1, t->scan32);
    if (r != VD_OK) return r;
    k_range_compact<<<grid_blocks(t, all, 256), 256, 0, s>>>(t->d_sorted.p, all, t->d_flags.p, t->d_pos.p,
                                                             t->d_bx_items.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
    VD_CK(t, cudaMemsetAsync(t->d_bx_sizes.p, 0, 3 * n * sizeof(int32_t), s));
    A.cursor = t->d_ctl.p + kCtlCursor;
    A.begin = begin;
    A.sizes = t->d_bx_sizes.p;
    std::vector<uint32_t> next;
    for (int tier = 0; tier < 3; ++tier) {
      if (tier > 0) {
        if (next.empty()) break;
        tier_at[tier] = tier == 1 ? nr : nr + tier_n[1];
        tier_n[tier] = (uint32_t)next.size();
        VD_CK(t, cudaMemcpyAsync(t->d_bx_items.p + tier_at[tier], next.data(), next.size() * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, s));
      }
      r = run_tier(0, tier);
      if (r != VD_OK) return r;
      VD_CK(t, cudaMemcpyAsync(sz.data(), t->d_bx_sizes.p, 3 * n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      VD_CK(t, cudaStreamSynchronize(s));
      next.clear();
      for (size_t k = 0; k < n; ++k)
        if (sz[3 * k] < 0) next.push_back((uint32_t)(begin + k));
    }
    for (uint32_t c : next) host_cells.push_back(c);
  }
  for (size_t c : host_cells) {
    int32_t nv = 0, nf = 0, nh = 0;
    r = vd_tess_get_cell(t, c, &nv, &nf, &nh, nullptr, nullptr, nullptr, nullptr);
    if (r != VD_OK) return r;
    const size_t k = c - begin;
    sz[3 * k] = nv;
    sz[3 * k + 1] = nf;
    sz[3 * k + 2] = nh;
  }
  v_off[0] = f_off[0] = h_off[0] = 0;
  for (size_t k = 0; k < n; ++k) {
    v_off[k + 1] = v_off[k] + sz[3 * k];
    f_off[k + 1] = f_off[k] + sz[3 * k + 1];
    h_off[k + 1] = h_off[k] + sz[3 * k + 2];
  }
  if (!fill) return VD_OK;
  if (device) {
    const size_t tv = (size_t)v_off[n], tf = (size_t)f_off[n], th = (size_t)h_off[n];
    VD_CK(t, t->d_bx_off.ensure(3 * (n + 1), s));
    VD_CK(t, t->d_bx_v.ensure(std::max<size_t>(3 * tv, 1), s));
    VD_CK(t, t->d_bx_fc.ensure(std::max<size_t>(tf, 1), s));
    VD_CK(t, t->d_bx_fn.ensure(std::max<size_t>(tf, 1), s));
    VD_CK(t, t->d_bx_fi.ensure(std::max<size_t>(th, 1), s));
    static_assert(sizeof(long long) == sizeof(int64_t), "offsets are 64-bit");
    VD_CK(t, cudaMemcpyAsync(t->d_bx_off.p, v_off, (n + 1) * 8, cudaMemcpyHostToDevice, s));
    VD_CK(t, cudaMemcpyAsync(t->d_bx_off.p + (n + 1), f_off, (n + 1) * 8, cudaMemcpyHostToDevice, s));
    VD_CK(t, cudaMemcpyAsync(t->d_bx_off.p + 2 * (n + 1), h_off, (n + 1) * 8, cudaMemcpyHostToDevice, s));
    A.voff = t->d_bx_off.p;
    A.foff = t->d_bx_off.p + (n + 1);
    A.hoff = t->d_bx_off.p + 2 * (n + 1);
    A.verts = t->d_bx_v.p;
    A.fc = t->d_bx_fc.p;
    A.fi = t->d_bx_fi.p;
    A.fn = t->d_bx_fn.p;
    A.sizes = nullptr;
    // a cell writes in the first tier that holds it (the rebuild is the same
    // in every tier, so the sizes agree with pass 0's)
    for (int tier = 0; tier < 3; ++tier) {
      if (tier_n[tier] == 0) continue;
      r = run_tier(1, tier);
      if (r != VD_OK) return r;
    }
    if (tv) VD_CK(t, cudaMemcpyAsync(vertices, t->d_bx_v.p, 3 * tv * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (tf) {
      VD_CK(t, cudaMemcpyAsync(face_counts, t->d_bx_fc.p, tf * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      VD_CK(t, cudaMemcpyAsync(face_neighbors, t->d_bx_fn.p, tf * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    }
    if (th) VD_CK(t, cudaMemcpyAsync(face_indices, t->d_bx_fi.p, th * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    VD_CK(t, cudaStreamSynchronize(s));
  }
  // the cells left to get_cell write straight into their slots
  for (size_t c : host_cells) {
    const size_t k = c - begin;
    int32_t nv = 0, nf = 0, nh = 0;
    r = vd_tess_get_cell(t, c, &nv, &nf, &nh, vertices + 3 * v_off[k], face_counts + f_off[k],
                         face_indices + h_off[k], face_neighbors + f_off[k]);
    if (r != VD_OK) return r;
  }
  return VD_OK;
}

int vd_tess_device_results(vd_tess* t, const double** d_volume, const double** d_centroid3,
                           const int32_t** d_n_faces) {
  int r = check_ready(t);
  if (r != VD_OK) return r;
  if (d_volume) *d_volume = t->d_vol.p;
  if (d_centroid3) *d_centroid3 = t->d_cen.p;
  if (d_n_faces) *d_n_faces = t->d_nf.p;
  return VD_OK;
}

int vd_tess_device_neighbors(vd_tess* t, const int64_t** d_offsets, const int32_t** d_ids, const double** d_areas,
                             int64_t* total) {
  int r = check_ready(t);
  if (r != VD_OK) return r;
  r = ensure_csr(t);
  if (r != VD_OK) return r;
  const size_t n = t->ncells;
  const size_t tot = (size_t)t->csr_total;
  cudaStream_t s = t->stream;
  VD_CK(t, t->d_csr_ids.ensure(tot, t->stream));
  VD_CK(t, t->d_csr_area.ensure(tot, t->stream));
  if (n && tot) {
    const int blocks = grid_blocks(t, n * 32, 256);
    k_csr_gather<<<blocks, 256, 0, s>>>(t->d_nf.p, n, t->d_csr_off.p, t->fout, t->d_fnb.p, t->d_farea.p,
                                        t->d_pool_fnb.p, t->d_pool_area.p, t->d_pool_off.p, t->d_csr_ids.p,
                                        t->d_csr_area.p);
    g_launches++;
    VD_CK(t, cudaGetLastError());
  }
  VD_CK(t, cudaStreamSynchronize(s));
  if (d_offsets) *d_offsets = reinterpret_cast<const int64_t*>(t->d_csr_off.p);
  if (d_ids) *d_ids = t->d_csr_ids.p;
  if (d_areas) *d_areas = t->d_csr_area.p;
  if (total) *total = t->csr_total;
  return VD_OK;
}

int vd_tess_stream(vd_tess* t, void** stream) {
  if (!t || !stream) return VD_EINVAL;
  *stream = (void*)t->stream;
  return VD_OK;
}

int vd_tess_timings(vd_tess* t, float* ms4) {
  if (!t || !ms4) return VD_EINVAL;
  memcpy(ms4, t->timings, sizeof(t->timings));
  return VD_OK;
}

int vd_tess_counters(vd_tess* t, uint64_t* out8) {
  if (!t || !out8) return VD_EINVAL;
  if (!t->instrument) return fail(t, VD_ESTATE, "counters need vd_tess_set_instrumentation(t, 1)");
  for (int k = 0; k < kNumCounters; ++k) out8[k] = t->counters[k];
  return VD_OK;
}

int vd_tess_fallback_counts(vd_tess* t, uint64_t* out2) {
  if (!t || !out2) return VD_EINVAL;
  out2[0] = t->fallback[0];
  out2[1] = t->fallback[1];
  return VD_OK;
}

int vd_launch_count(uint64_t* n) {
  if (!n) return VD_EINVAL;
  *n = g_launches.load();
  return VD_OK;
}

int vd_host_alloc(size_t bytes, void** ptr) {
  if (!ptr) return VD_EINVAL;
  cudaError_t e = cudaHostAlloc(ptr, std::max<size_t>(bytes, 1), cudaHostAllocDefault);
  if (e != cudaSuccess) return fail(nullptr, VD_ENOMEM, "cudaHostAlloc: %s", cudaGetErrorString(e));
  return VD_OK;
}

int vd_host_free(void* ptr) {
  if (ptr) cudaFreeHost(ptr);
  return VD_OK;
}

}  // extern "C"
