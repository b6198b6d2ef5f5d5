// vd_binning.cuh -- device kernels around the clip kernel: wall filtering and
// stream compaction (Tessellation::set_generators, tessellation.rs:43-67),
// binning by counting sort (Algorithm3DGrid::set_generators,
// algo_3d_grid.rs:111-130), scans, the CSR export of per-face results and
// the Lloyd update (Tessellation::relax, tessellation.rs:482-495).
//
// All of these are HBM-bound integer/byte work: coalesced loads, one pass per
// step, grids sized from the SM count.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "vd_common.cuh"

namespace vd {
// internal linkage: every translation unit that launches these gets its own copy
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// ---- scan (exclusive) -------------------------------------------------------
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* total, T* sh) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    T s = lane < (kScanThreads / 32) ? sh[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < (kScanThreads / 32)) sh[lane] = s;
  }
  __syncthreads();
  const T before = w > 0 ? sh[w - 1] : T(0);
  *total = sh[kScanThreads / 32 - 1];
  __syncthreads();
  return before + x - v;
}

template <typename Tin, typename T>
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const Tin* in, T* out, size_t n, T* sums) {
  __shared__ T sh[kScanThreads / 32];
  const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  T v[kScanItems];
  T s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? (T)in[base + k] : T(0);
    s += v[k];
  }
  T total;
  T ex = block_excl_scan<T>(s, &total, sh);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = ex;
    ex += v[k];
  }
  if (threadIdx.x == 0 && sums) sums[blockIdx.x] = total;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_scan_add(T* out, size_t n, const T* offs) {
  const T add = offs[blockIdx.x];
  const size_t base = (size_t)blockIdx.x * kScanTile;
  for (int k = threadIdx.x; k < kScanTile; k += kScanThreads)
    if (base + k < n) out[base + k] += add;
}

// ---- walls ------------------------------------------------------------------
// WallGeometry::contains of each wall kind (wall_3d.rs:31-36, 73-78, 132-143,
// 202-214, 293-309, 691-701), in the reference's arithmetic order; also run on
// the host by set_generator (host code is built with -ffp-contract=off)
__host__ __device__ __forceinline__ bool wall_contains(const Wall& w, const double* planes, double x, double y, double z) {
  const double dx = x - w.a[0], dy = y - w.a[1], dz = z - w.a[2];
  switch (w.kind) {
    case kWallPlane:
      return (dx * w.n[0] + dy * w.n[1] + dz * w.n[2]) >= 0.0;
    case kWallSphere:
      return (dx * dx + dy * dy + dz * dz) <= w.r * w.r;
    case kWallCylinder: {
      const double dot = dx * w.n[0] + dy * w.n[1] + dz * w.n[2];
      const double px = dx - dot * w.n[0], py = dy - dot * w.n[1], pz = dz - dot * w.n[2];
      return (px * px + py * py + pz * pz) <= w.r * w.r;
    }
    case kWallCone: {
      const double h = dx * w.n[0] + dy * w.n[1] + dz * w.n[2];
      const double px = dx - h * w.n[0], py = dy - h * w.n[1], pz = dz - h * w.n[2];
      const double r = sqrt(px * px + py * py + pz * pz);
      return h >= 0.0 && r <= h * w.ta;
    }
    case kWallTorus: {
      const double dot = dx * w.n[0] + dy * w.n[1] + dz * w.n[2];
      const double px = dx - dot * w.n[0], py = dy - dot * w.n[1], pz = dz - dot * w.n[2];
      const double q = sqrt(px * px + py * py + pz * pz) - w.r;
      return sqrt(q * q + dot * dot) <= w.r2;
    }
    default:
      for (int k = 0; k < w.np; ++k) {
        const double* pl = planes + 6 * (w.p0 + k);
        const double ex = x - pl[0], ey = y - pl[1], ez = z - pl[2];
        if (ex * pl[3] + ey * pl[4] + ez * pl[5] > 0.0) return false;
      }
      return true;
  }
}

struct WallSet {
  int n;
  Wall w[kMaxWalls];
  const double* planes;
};

__global__ void k_wall_flags(const double* __restrict__ in, size_t n, const WallSet ws, uint32_t* flags) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double x = in[3 * i], y = in[3 * i + 1], z = in[3 * i + 2];
    bool ok = true;
    for (int k = 0; k < ws.n && ok; ++k) ok = wall_contains(ws.w[k], ws.planes, x, y, z);
    flags[i] = ok ? 1u : 0u;
  }
}

__global__ void k_compact3(const double* __restrict__ in, size_t n, const uint32_t* flags, const uint32_t* pos,
                           double* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if (flags[i]) {
      const size_t o = pos[i];
      out[3 * o] = in[3 * i];
      out[3 * o + 1] = in[3 * i + 1];
      out[3 * o + 2] = in[3 * i + 2];
    }
  }
}

// ---- random generators ------------------------------------------------------
// SplitMix64 (Steele, Lea & Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014) as a counter-based generator: draw k of a seed is
// the SplitMix64 output mix of seed + (k + 1) * 0x9e3779b97f4a7c15, so every
// candidate's coordinates are fixed by (seed, index) alone.
__host__ __device__ __forceinline__ uint64_t splitmix64_at(uint64_t seed, uint64_t k) {
  uint64_t z = seed + (k + 1) * 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Candidate a of Tessellation::random_generators (tessellation.rs:96-121):
// coordinate c = min[c] + u * (max[c] - min[c]), u = (draw 3a + c >> 11) * 2^-53
// in [0, 1) (the 53-bit mapping of rand's Standard f64); flagged when every
// wall contains it.
__global__ void k_random_candidates(uint64_t seed, uint64_t a0, size_t n, const Grid g, const WallSet ws,
                                    double* __restrict__ out, uint32_t* flags) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint64_t a = a0 + i;
    double p[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double u = (double)(splitmix64_at(seed, 3 * a + c) >> 11) * 0x1p-53;
      p[c] = g.bmin[c] + u * (g.bmax[c] - g.bmin[c]);
    }
    bool ok = true;
    for (int k = 0; k < ws.n && ok; ++k) ok = wall_contains(ws.w[k], ws.planes, p[0], p[1], p[2]);
    out[3 * i] = p[0];
    out[3 * i + 1] = p[1];
    out[3 * i + 2] = p[2];
    flags[i] = ok ? 1u : 0u;
  }
}

// k_compact3 keeping only the flagged rows ranked below `limit`
__global__ void k_compact3_first(const double* __restrict__ in, size_t n, const uint32_t* flags,
                                 const uint32_t* pos, uint32_t limit, double* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if (flags[i] && pos[i] < limit) {
      const size_t o = pos[i];
      out[3 * o] = in[3 * i];
      out[3 * o + 1] = in[3 * i + 1];
      out[3 * o + 2] = in[3 * i + 2];
    }
  }
}

// ---- binning ----------------------------------------------------------------
__device__ __forceinline__ uint32_t axis_index(double v, double lo, double scale, double limit) {
  double t = (v - lo) * scale;  // clamp(0, limit) then `as usize` (NaN -> 0)
  if (t < 0.0) t = 0.0;
  if (t > limit) t = limit;
  return t > 0.0 ? (uint32_t)t : 0u;
}

// get_bin_index (algo_3d_grid.rs:98-107)
__device__ __forceinline__ uint32_t bin_index(const Grid& g, double x, double y, double z) {
  const uint32_t ix = axis_index(x, g.bmin[0], g.scale[0], g.limit[0]);
  const uint32_t iy = axis_index(y, g.bmin[1], g.scale[1], g.limit[1]);
  const uint32_t iz = axis_index(z, g.bmin[2], g.scale[2], g.limit[2]);
  return ix + iy * (uint32_t)g.n[0] + iz * (uint32_t)g.n[0] * (uint32_t)g.n[1];
}

__global__ void k_bin_count(const double* __restrict__ gen, size_t n, const Grid g, uint32_t* __restrict__ bin_of,
                            uint32_t* counts) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t b = bin_index(g, gen[3 * i], gen[3 * i + 1], gen[3 * i + 2]);
    bin_of[i] = b;
    atomicAdd(&counts[b], 1u);
  }
}

__global__ void k_bin_scatter(const uint32_t* __restrict__ bin_of, size_t n, uint32_t* cursor,
                              uint32_t* __restrict__ ids) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    ids[atomicAdd(&cursor[bin_of[i]], 1u)] = (uint32_t)i;
}

// occ[w] bit j = 1 when bin 32 w + j has members: the walk's test for an
// empty bin without reading bin_start (on a sparse grid the bin table is
// large and mostly empty; the bit map is 1/32 of it and stays in L2)
__global__ void k_bin_occupancy(const uint32_t* __restrict__ start, size_t nbins, uint32_t* __restrict__ occ) {
  const size_t nw = (nbins + 31) / 32;
  for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (size_t)gridDim.x * blockDim.x) {
    uint32_t m = 0;
    const size_t b0 = 32 * w;
    uint32_t prev = start[b0];
    for (int j = 0; j < 32 && b0 + j < nbins; ++j) {
      const uint32_t next = start[b0 + j + 1];
      if (next > prev) m |= 1u << j;
      prev = next;
    }
    occ[w] = m;
  }
}

constexpr uint32_t kSmallBin = 16;

// The atomic scatter leaves members in arbitrary order; the reference pushes
// them in ascending id order.  Small bins are insertion-sorted in place, big
// ones are listed for k_bin_sort_big.
__global__ void k_bin_fix(const uint32_t* __restrict__ start, size_t nbins, uint32_t* ids, uint32_t* big_list,
                          unsigned int* big_count) {
  for (size_t b = (size_t)blockIdx.x * blockDim.x + threadIdx.x; b < nbins; b += (size_t)gridDim.x * blockDim.x) {
    const uint32_t s = start[b], e = start[b + 1];
    const uint32_t c = e - s;
    if (c <= 1) continue;
    if (c > kSmallBin) {
      big_list[atomicAdd(big_count, 1u)] = (uint32_t)b;
      continue;
    }
    for (uint32_t k = s + 1; k < e; ++k) {  // insertion sort, in place
      const uint32_t x = ids[k];
      uint32_t j = k;
      while (j > s && ids[j - 1] > x) {
        ids[j] = ids[j - 1];
        --j;
      }
      ids[j] = x;
    }
  }
}

constexpr int kBigSortThreads = 256;
constexpr int kBigSortChunk = 4096;

// One block per big bin: bitonic-sort chunks of 4096 in shared memory, then
// merge runs by rank (ids are unique, so a rank is a binary search).
__global__ void __launch_bounds__(kBigSortThreads)
    k_bin_sort_big(const uint32_t* __restrict__ start, const uint32_t* list, const unsigned int* count,
                   uint32_t* ids, uint32_t* tmp) {
  __shared__ uint32_t sh[kBigSortChunk];
  const unsigned nl = *count;
  for (unsigned li = blockIdx.x; li < nl; li += gridDim.x) {
    const uint32_t b = list[li];
    const uint32_t s = start[b], c = start[b + 1] - s;
    for (uint32_t c0 = 0; c0 < c; c0 += kBigSortChunk) {
      const uint32_t m = min((uint32_t)kBigSortChunk, c - c0);
      uint32_t p2 = 1;
      while (p2 < m) p2 <<= 1;
      for (uint32_t k = threadIdx.x; k < p2; k += blockDim.x) sh[k] = k < m ? ids[s + c0 + k] : 0xffffffffu;
      __syncthreads();
      for (uint32_t size = 2; size <= p2; size <<= 1) {
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
          for (uint32_t k = threadIdx.x; k < p2; k += blockDim.x) {
            const uint32_t j = k ^ stride;
            if (j > k) {
              const bool up = (k & size) == 0;
              const uint32_t a = sh[k], bb = sh[j];
              if ((a > bb) == up) {
                sh[k] = bb;
                sh[j] = a;
              }
            }
          }
          __syncthreads();
        }
      }
      for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) ids[s + c0 + k] = sh[k];
      __syncthreads();
    }
    uint32_t* src = ids + s;
    uint32_t* dst = tmp + s;
    for (uint32_t w = kBigSortChunk; w < c; w <<= 1) {
      for (uint32_t k = threadIdx.x; k < c; k += blockDim.x) {
        const uint32_t run = k / (2 * w);
        const uint32_t lo = run * 2 * w;
        const uint32_t mid = min(lo + w, c), hi = min(lo + 2 * w, c);
        const uint32_t x = src[k];
        uint32_t olo, ohi, rank_self;
        if (k < mid) {
          olo = mid;
          ohi = hi;
          rank_self = k - lo;
        } else {
          olo = lo;
          ohi = mid;
          rank_self = k - mid;
        }
        uint32_t a = olo, e = ohi;  // count of elements < x in the other run
        while (a < e) {
          const uint32_t md = (a + e) >> 1;
          if (src[md] < x) a = md + 1;
          else e = md;
        }
        dst[lo + rank_self + (a - olo)] = x;
      }
      __syncthreads();
      uint32_t* t = src;
      src = dst;
      dst = t;
    }
    if (src != ids + s)
      for (uint32_t k = threadIdx.x; k < c; k += blockDim.x) ids[s + k] = src[k];
    __syncthreads();
  }
}

__global__ void k_gather_sorted(const uint32_t* __restrict__ ids, const double* __restrict__ gen, size_t n,
                                SortedGen* __restrict__ out) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const uint32_t i = ids[k];
    SortedGen s;
    s.x = gen[3 * (size_t)i];
    s.y = gen[3 * (size_t)i + 1];
    s.z = gen[3 * (size_t)i + 2];
    s.id = (long long)i;
    out[k] = s;
  }
}

// ---- results ----------------------------------------------------------------
__global__ void k_nfaces_to_i64(const int32_t* __restrict__ nf, size_t n, long long* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = nf[i] > 0 ? nf[i] : 0;
}

__global__ void k_csr_gather(const int32_t* __restrict__ nf, size_t n, const long long* __restrict__ off, int fout,
                             const int32_t* __restrict__ fnb, const double* __restrict__ farea,
                             const int32_t* __restrict__ pool_fnb, const double* __restrict__ pool_farea,
                             const long long* __restrict__ pool_off, int32_t* __restrict__ out_ids,
                             double* __restrict__ out_area) {
  // one warp per cell: lanes copy the faces
  const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t i = gw; i < n; i += nw) {
    const int c = nf[i];
    if (c <= 0) continue;
    const long long o = off[i];
    const bool pooled = c > fout;
    // a pooled cell without slots (-1) has nothing to copy; the host reports
    // pool overflow as an error before results can be read
    if (pooled && pool_off[i] < 0) continue;
    for (int f = lane; f < c; f += 32) {
      const size_t src = pooled ? (size_t)pool_off[i] + f : i * (size_t)fout + f;
      if (out_ids) out_ids[o + f] = pooled ? pool_fnb[src] : fnb[src];
      if (out_area) out_area[o + f] = pooled ? pool_farea[src] : farea[src];
    }
  }
}

// Tessellation::relax: new generator = centroid, or the old position when the
// cell is empty (tessellation.rs:483-492)
__global__ void k_relax(const double* __restrict__ gen, const int32_t* __restrict__ nverts,
                        const double* __restrict__ cen, size_t n, double* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const bool empty = nverts[i] == 0;
    const double* src = empty ? gen : cen;
    out[3 * i] = src[3 * i];
    out[3 * i + 1] = src[3 * i + 1];
    out[3 * i + 2] = src[3 * i + 2];
  }
}

// ---- cell-id ranges (calculate_range, calculate_strided) ---------------------
// flags[k] = 1 when the generator at bin-order position k has an id in
// [begin, end) whose chunk index (id - begin) / chunk is phase modulo stride;
// the scan of the flags then lists those cells in bin order, so a shard's
// warps still walk neighbouring cells one after another.
__global__ void k_range_flags(const SortedGen* __restrict__ sorted, size_t n, long long begin, long long end,
                              long long chunk, long long stride, long long phase, uint32_t* __restrict__ flags) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const long long id = sorted[k].id;
    flags[k] = (id >= begin && id < end && ((id - begin) / chunk) % stride == phase) ? 1u : 0u;
  }
}

__global__ void k_range_compact(const SortedGen* __restrict__ sorted, size_t n, const uint32_t* __restrict__ flags,
                                const uint32_t* __restrict__ pos, uint32_t* __restrict__ list) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    if (flags[k]) list[pos[k]] = (uint32_t)sorted[k].id;
}

// flags[i] = mask[i] != 0, and the flagged ids compacted in id order
__global__ void k_nonzero_flags(const uint32_t* __restrict__ mask, size_t n, uint32_t* __restrict__ flags) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    flags[i] = mask[i] != 0u ? 1u : 0u;
}

__global__ void k_compact_ids(const uint32_t* __restrict__ flags, const uint32_t* __restrict__ pos, size_t n,
                              uint32_t* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (flags[i]) out[pos[i]] = (uint32_t)i;
}

// cells outside a computed range read as empty (volume 0, centroid 0, no faces)
__global__ void k_clear_cells(size_t n, double* __restrict__ vol, double* __restrict__ cen,
                              int32_t* __restrict__ nfaces, int32_t* __restrict__ nverts) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    vol[i] = 0.0;
    cen[3 * i] = 0.0;
    cen[3 * i + 1] = 0.0;
    cen[3 * i + 2] = 0.0;
    nfaces[i] = 0;
    nverts[i] = 0;
  }
}

}  // namespace
}  // namespace vd
