// vd_clip.cuh -- warp-per-cell Voronoi cell construction (FP64, bit-exact path).
//
// One warp owns one cell.  The convex polytope (vertex list + face loops, the
// layout of Cell3DFaces, cell_3d_faces.rs:24-34) lives in a per-warp
// WarpPoly: shared memory on the fast path, a global-memory slice on the
// large-capacity pass.  Every step of Cell3DFaces::clip_with_scratch
// (cell_3d_faces.rs:288-503) is done warp-parallel but produces exactly the
// reference's output order:
//   * vertex classification: one vertex per lane, ballots give all-in/all-out;
//   * kept vertices: ballot-compacted in their original order;
//   * crossing edges: ballot-compacted in face-walk order; the first
//     occurrence of each (min,max) edge key (match.any) creates the
//     intersection vertex, later ones reuse it -- the reference's
//     intersection_map semantics, including its numbering;
//   * face rewiring: per-position emit counts (0/1/2) and a warp scan give
//     every surviving entry its slot; faces with < 3 entries are dropped;
//   * the lid: segments between consecutive intersection vertices, a
//     last-writer-wins lid_map, and one lane following the chain.
// Arithmetic is written in the reference's evaluation order; the translation
// unit is compiled with -fmad=false so no multiply-add is fused, and division
// and square root are IEEE correctly rounded, so every double equals the
// reference's.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "vd_common.cuh"
#include "vd_wall.cuh"

namespace vd {

constexpr unsigned kFull = 0xffffffffu;

template <int V, int F, int H, int CC, int NC, int SC, typename VIdT, typename FIdT, typename KeyT,
          typename CIdT, bool kCount, bool kMixed, typename PosT = uint16_t, typename DelT = int16_t>
struct PolyCfg {
  static constexpr bool COUNT = kCount;  // maintain the algorithmic event counters
  static constexpr bool MIXED = kMixed;  // FP32 classification under an error bound
  static constexpr int VCAP = V;   // vertices
  static constexpr int FCAP = F;   // faces
  static constexpr int HCAP = H;   // flattened face-index entries
  static constexpr int CCAP = CC;  // crossing positions per clip
  static constexpr int NCAP = NC;  // new (intersection) vertices per clip
  static constexpr int SCAP = SC;  // lid segments per clip
  using VId = VIdT;
  using FId = FIdT;
  using Key = KeyT;  // (min, max) vertex pair of an edge
  using CId = CIdT;  // crossing index
  using Pos = PosT;  // face-entry position (and triangle prefix)
  using Del = DelT;  // difference of two positions
  static constexpr int KSHIFT = 8 * (int)sizeof(VIdT);
  static constexpr unsigned VNONE = (unsigned)(VIdT)~(VIdT)0;
  static constexpr unsigned FNONE = (unsigned)(FIdT)~(FIdT)0;
  static_assert(V < (int)VNONE, "vertex ids must leave room for the none marker");
  static_assert(F < (int)FNONE, "face ids must leave room for the none marker");
};

// Fast path: sized from the oracle's distribution (max 72 vertices, 38 faces,
// 216 face entries over 7.5M uniform-input polytopes); anything larger goes
// to the large-capacity pass.
// With at most 32 crossing positions per clip, each new vertex stays in the
// register of the lane that discovered it until the vertex list is rebuilt.
using FastCfg = PolyCfg<96, 48, 288, 32, 32, 32, uint8_t, uint8_t, uint16_t, uint8_t, false, false>;
// the same with the event counters (instrumented runs)
using FastCfgCount = PolyCfg<96, 48, 288, 32, 32, 32, uint8_t, uint8_t, uint16_t, uint8_t, true, false>;
// mixed precision: same capacities, FP32 generator-relative copies of the vertices
using MixedCfg = PolyCfg<96, 48, 288, 32, 32, 32, uint8_t, uint8_t, uint16_t, uint8_t, false, true>;
using MixedCfgCount = PolyCfg<96, 48, 288, 32, 32, 32, uint8_t, uint8_t, uint16_t, uint8_t, true, true>;
// Medium tier (shared memory, 2 warps per block): cells whose polytope
// outgrew the fast capacities -- typical of dense clustered inputs, where
// the reference's bin-order walk clips a cell with thousands of candidates.
using MedCfg = PolyCfg<224, 112, 672, 128, 64, 64, uint8_t, uint8_t, uint16_t, uint8_t, true, false>;
// the same without the event counters (uninstrumented single tessellations)
using MedCfgNC = PolyCfg<224, 112, 672, 128, 64, 64, uint8_t, uint8_t, uint16_t, uint8_t, false, false>;
// Large-capacity pass (global-memory storage): vertex ids stay u16 like the
// reference's face_indices (cell_3d_faces.rs:31).
using BigCfg = PolyCfg<2048, 512, 6144, 1024, 512, 512, uint16_t, uint16_t, uint32_t, uint16_t, true, false>;
// Huge tier (global memory, one thread block per cell, vd_clip_block.cuh):
// cells adjacent to thousands of others, such as the centre of generators on a
// sphere.  Vertex ids stay u16 like the reference's face_indices; positions
// are 32-bit.  No event counters.
using HugeCfg = PolyCfg<65534, 32767, 196608, 16384, 8192, 8192, uint16_t, uint16_t, uint32_t, uint16_t, false, false,
                        uint32_t, int32_t>;

// the new ids of the two ends of one face position's edge
template <typename V>
struct alignas(2 * sizeof(V)) VPair {
  V s, e;
};

struct PolyState;

template <class C>
struct alignas(16) WarpPoly {
  using State = PolyState;
  static constexpr bool kExport = true;  // vertices in the reference's order: exportable
  double vx[C::VCAP], vy[C::VCAP], vz[C::VCAP];
  // plain path: the FP64 signed distances of the current clip
  double dist[C::MIXED ? 1 : C::VCAP];
  // mixed path: FP32 copies of the vertices relative to the generator
  float ux[C::MIXED ? C::VCAP : 1], uy[C::MIXED ? C::VCAP : 1], uz[C::MIXED ? C::VCAP : 1];
  // new vertices awaiting the rebuilt list (only when a clip can have more
  // than 32 crossings; otherwise they wait in registers)
  double tx[C::CCAP > 32 ? C::NCAP : 1], ty[C::CCAP > 32 ? C::NCAP : 1], tz[C::CCAP > 32 ? C::NCAP : 1];
  unsigned long long cnt[C::COUNT ? kNumCounters : 1];
  int32_t fn[2][C::FCAP];
  typename C::Pos E[C::HCAP + 1];
  typename C::Pos fs[2][C::FCAP + 1];
  typename C::Pos fns[C::FCAP];
  typename C::Pos cpos[C::CCAP];
  typename C::Key ckey[C::CCAP];
  typename C::VId cid[C::CCAP];
  typename C::VId fi[2][C::HCAP];
  typename C::FId pf[2][C::HCAP];
  typename C::VId fe[C::HCAP];    // per clip: end vertex of each position's edge
  typename C::CId cidx[C::HCAP];  // per clip: crossing index of a crossing position
  typename C::CId fcr[C::FCAP];   // per clip: index of each face's first crossing
  VPair<typename C::VId> pve[C::HCAP];  // per clip: new ids of each position's edge ends (or none)
  typename C::Del fdel[C::FCAP];          // per clip: new entry offset of a face minus its first position's E
  uint8_t cand_e[32];             // walk: search-order entry (lane) of each candidate of a round
  typename C::FId fnew[C::FCAP];
  typename C::VId o2n[C::VCAP];
  typename C::VId lidmap[C::VCAP];
  typename C::VId sega[C::SCAP], segb[C::SCAP];
};

struct PolyState {
  int nv, nf, nh, cb;
  double umax;  // mixed path: bound on |v - g| (max norm) over the vertices
};

__device__ __forceinline__ bool state_empty(const PolyState& S) { return S.nv == 0; }

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ int warp_incl_scan(int x) {
  const unsigned lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(kFull, x, o);
    if ((int)lane >= o) x += y;
  }
  return x;
}

__device__ __forceinline__ double warp_max(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(kFull, x, o));
  return x;
}

// The largest of the lanes' values, each a non-negative double or NaN (NaN
// counts as 0, as fmax and the reference's `d2 > max` comparison treat it).
// Non-negative doubles order like their bit patterns as unsigned integers, so
// two 32-bit reductions give exactly fmax's result.
__device__ __forceinline__ double sp_warp_max_nonneg(double x) {
  const unsigned long long b = (x >= 0.0) ? (unsigned long long)__double_as_longlong(x) : 0ull;
  const unsigned hi = __reduce_max_sync(kFull, (unsigned)(b >> 32));
  const unsigned lo = __reduce_max_sync(kFull, (unsigned)(b >> 32) == hi ? (unsigned)b : 0u);
  return __longlong_as_double((long long)(((unsigned long long)hi << 32) | lo));
}

__device__ __forceinline__ double clamp01(double t) {
  // f64::clamp(0.0, 1.0); NaN passes through
  if (t < 0.0) return 0.0;
  if (t > 1.0) return 1.0;
  return t;
}

template <class C>
__device__ __forceinline__ void cnt_add(WarpPoly<C>& P, int k, unsigned long long v) {
  if constexpr (C::COUNT) {
    if (lane_id() == 0) P.cnt[k] += v;
  }
}

// Cell3DFaces::new (cell_3d_faces.rs:37-74): the box, faces z-, z+, y-, y+,
// x-, x+ with ids box_side (bounds/mod.rs:21-22).
template <class C>
__device__ void poly_init_box(WarpPoly<C>& P, PolyState& S, const Grid& g, double gx, double gy, double gz) {
  const unsigned lane = lane_id();
  if (lane < 8) {
    const unsigned hx = (lane == 1 || lane == 2 || lane == 5 || lane == 6);
    const unsigned hy = (lane == 2 || lane == 3 || lane == 6 || lane == 7);
    const unsigned hz = lane >= 4;
    P.vx[lane] = hx ? g.bmax[0] : g.bmin[0];
    P.vy[lane] = hy ? g.bmax[1] : g.bmin[1];
    P.vz[lane] = hz ? g.bmax[2] : g.bmin[2];
  }
  // face loops 3210 4567 0154 2376 0473 1265 packed as nibbles, lane = entry
  if (lane < 24) {
    const unsigned long long lo = 0x6732451076540123ull, hi = 0x56213740ull;
    const unsigned idx = (unsigned)((lane < 16 ? lo >> (4 * lane) : hi >> (4 * (lane - 16))) & 0xFull);
    P.fi[0][lane] = (typename C::VId)idx;
    P.pf[0][lane] = (typename C::FId)(lane >> 2);
  }
  if (lane < 7) P.fs[0][lane] = (typename C::Pos)(4 * lane);
  // face ids z-, z+, y-, y+, x-, x+ = box_side(axis, is_max) = -1 - (2*axis + is_max)
  if (lane < 6) P.fn[0][lane] = -1 - (2 * (2 - (int)(lane >> 1)) + (int)(lane & 1));
  S.nv = 8;
  S.nf = 6;
  S.nh = 24;
  S.cb = 0;
  S.umax = 0.0;
  if constexpr (C::MIXED) {
    double m = 0.0;
    if (lane < 8) {
      const float fx = (float)(P.vx[lane] - gx), fy = (float)(P.vy[lane] - gy), fz = (float)(P.vz[lane] - gz);
      P.ux[lane] = fx;
      P.uy[lane] = fy;
      P.uz[lane] = fz;
      m = fmax(fabs((double)fx), fmax(fabs((double)fy), fabs((double)fz)));
    }
    S.umax = warp_max(m) * (1.0 + 0x1p-20);
  }
  __syncwarp();
}

// max_radius_sq (cell_3d_faces.rs:271-286)
template <class C>
__device__ double poly_max_radius_sq(const WarpPoly<C>& P, const PolyState& S, double gx, double gy,
                                     double gz) {
  double m = 0.0;
  for (int v = lane_id(); v < S.nv; v += 32) {
    double dx = P.vx[v] - gx;
    double dy = P.vy[v] - gy;
    double dz = P.vz[v] - gz;
    double d2 = dx * dx + dy * dy + dz * dz;
    m = fmax(m, d2);
  }
  return warp_max(m);
}

// clip_with_scratch (cell_3d_faces.rs:288-503).  All lanes call it with the
// same (uniform) arguments.  *r2 gets the max squared distance of the new
// vertex set from (gx,gy,gz) when with_gen, else 0.
template <class C>
__device__ int warp_clip(WarpPoly<C>& P, PolyState& S, double px, double py, double pz, double nx,
                         double ny, double nz, int nbr, bool with_gen, double gx, double gy, double gz,
                         double* r2out) {
  using VId = typename C::VId;
  using FId = typename C::FId;
  const unsigned lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  const int nv = S.nv, nf = S.nf, nh = S.nh, cb = S.cb, nb = cb ^ 1;
  cnt_add(P, kCntClips, 1);
  cnt_add(P, kCntClassified, (unsigned long long)nv);

  // 1. signed distances and the 3-band flags (:302-326); o2n marks the
  //    vertices to keep (d <= 1e-9) until step 2 numbers them
  bool out = false, sin = false;
  if constexpr (!C::MIXED) {
    for (int v = lane; v < nv; v += 32) {
      double d = (P.vx[v] - px) * nx + (P.vy[v] - py) * ny + (P.vz[v] - pz) * nz;
      P.dist[v] = d;
      P.o2n[v] = d > kTol ? (VId)C::VNONE : (VId)0;
      out |= d > kTol;
      sin |= d < -kTol;
    }
  } else {
    // FP32 distance on generator-relative coordinates, d32 = u.n - c with
    // c = (p - g).n.  Forward error bound against the FP64 value
    // d64 = (v - p).n of the plain path (u = fl32(fl64(v - g))):
    //   |d32 - d64| <= 2^-21 (|u|_inf |n|_1 + |c| + sum_k |(p_k - g_k) n_k|) + 1e-30.
    // A vertex whose d32 lies within that bound of +-1e-9 is re-evaluated
    // with the plain path's FP64 formula, so every decision equals it.
    const double qx = px - gx, qy = py - gy, qz = pz - gz;
    const double c = qx * nx + qy * ny + qz * nz;
    const double qn = fabs(qx * nx) + fabs(qy * ny) + fabs(qz * nz);
    const double scale = S.umax * (fabs(nx) + fabs(ny) + fabs(nz)) + fabs(c);
    const double bound = 0x1p-21 * (scale + qn) + 1e-30;
    const bool fp32_ok = scale > 1e-24 && scale < 1e24;
    const float fnx = (float)nx, fny = (float)ny, fnz = (float)nz, fc = (float)c;
    const double hi_out = kTol + bound, lo_sin = -kTol - bound;
    const double band_lo = -kTol + bound, band_hi = kTol - bound;
    for (int v = lane; v < nv; v += 32) {
      bool o = false, si = false, exact = !fp32_ok;
      if (fp32_ok) {
        const double d32 = (double)(fmaf(P.ux[v], fnx, fmaf(P.uy[v], fny, P.uz[v] * fnz)) - fc);
        if (d32 > hi_out) o = true;
        else if (d32 < lo_sin) si = true;
        else exact = !(d32 >= band_lo && d32 <= band_hi);
      }
      if (exact) {
        const double d = (P.vx[v] - px) * nx + (P.vy[v] - py) * ny + (P.vz[v] - pz) * nz;
        o = d > kTol;
        si = d < -kTol;
      }
      P.o2n[v] = o ? (VId)C::VNONE : (VId)0;
      out |= o;
      sin |= si;
    }
  }
  if (!__any_sync(kFull, out)) {
    *r2out = 0.0;
    return kClipNoop;
  }
  if (!__any_sync(kFull, sin)) {
    S.nv = S.nf = S.nh = 0;
    *r2out = 0.0;
    return kClipEmpty;
  }
  cnt_add(P, kCntModifying, 1);
  __syncwarp();

  // 2. keep the inside vertices in order (:344-362)
  int nkept = 0;
  double r2 = 0.0;
  for (int b = 0; b < nv; b += 32) {
    const int v = b + lane;
    const bool k = v < nv && P.o2n[v] != C::VNONE;
    const unsigned m = __ballot_sync(kFull, k);
    if (v < nv) P.o2n[v] = k ? (VId)(nkept + __popc(m & lt)) : (VId)C::VNONE;
    if (k && with_gen) {
      double dx = P.vx[v] - gx;
      double dy = P.vy[v] - gy;
      double dz = P.vz[v] - gz;
      double d2 = dx * dx + dy * dy + dz * dz;
      r2 = fmax(r2, d2);
    }
    nkept += __popc(m);
  }
  if (with_gen) cnt_add(P, kCntKept, (unsigned long long)nkept);

  __syncwarp();

  // 3. one pass over the face positions (the face walk of :369-452): the
  //    edge's end vertex, the crossing positions in walk order, and the
  //    exclusive prefix E of the entries each position emits into the new
  //    faces: in->in 1 (end), in->out 1 (X), out->in 2 (X, end), out->out 0.
  //    A crossing is its face's first when no earlier crossing lies at or
  //    after the face's first position; step 7 finds a segment's partner
  //    through it.
  int ncross = 0;
  {
    int run = 0;
    int lastcross = -1;  // position of the last crossing of earlier chunks
    for (int b = 0; b < nh; b += 32) {
      const int p = b + lane;
      bool cr = false, si = false, ei = false;
      int f = 0, f0 = 0;
      unsigned s = 0, e = 0;
      if (p < nh) {
        f = P.pf[cb][p];
        f0 = P.fs[cb][f];
        s = P.fi[cb][p];
        // the edge's end: the next entry of the face loop ((i + 1) % count, :380)
        e = P.fi[cb][(p + 1 == P.fs[cb][f + 1]) ? f0 : p + 1];
        const VId os = P.o2n[s], oe = P.o2n[e];
        si = os != C::VNONE;
        ei = oe != C::VNONE;
        P.fe[p] = (VId)e;
        P.pve[p] = VPair<VId>{os, oe};
        cr = si != ei;
      }
      const unsigned m = __ballot_sync(kFull, cr);
      if (cr) {
        const int k = ncross + __popc(m & lt);
        const unsigned before = m & lt;
        const int prevp = before ? b + 31 - __clz(before) : lastcross;
        if (k < C::CCAP) {
          P.cpos[k] = (typename C::Pos)p;
          P.ckey[k] = (typename C::Key)(s < e ? (s << C::KSHIFT | e) : (e << C::KSHIFT | s));
          P.cidx[p] = (typename C::CId)k;
          if (prevp < f0) P.fcr[f] = (typename C::CId)k;
        }
      }
      if (m) lastcross = b + 31 - __clz(m);
      ncross += __popc(m);
      // emit counts are 1 (start inside) or 2 (out->in): the prefix is two
      // ballot populations
      const unsigned m1 = __ballot_sync(kFull, si);
      const unsigned m2 = __ballot_sync(kFull, !si && ei);
      if (p < nh) P.E[p] = (typename C::Pos)(run + __popc(m1 & lt) + 2 * __popc(m2 & lt));
      run += __popc(m1) + 2 * __popc(m2);
    }
    if (lane == 0) P.E[nh] = (typename C::Pos)run;
  }
  if (ncross > C::CCAP) return kClipOverflow;
  __syncwarp();

  // 4. intersection vertices: the first occurrence of an edge key creates the
  //    vertex (numbered in discovery order after the kept ones), repeats reuse
  //    it (the intersection_map lookups of :391-417 / :422-448)
  int nnew = 0;
  constexpr bool kRegX = C::CCAP <= 32;  // a single chunk: keep new vertices in registers
  double rx = 0.0, ry = 0.0, rz = 0.0;
  int rslot = -1;
  for (int b = 0; b < ncross; b += 32) {
    const int k = b + lane;
    const bool act = k < ncross;
    const unsigned key = act ? (unsigned)P.ckey[k] : (0xFFFF0000u | lane);
    const unsigned mm = __match_any_sync(kFull, key);
    const int leader = __ffs(mm) - 1;
    const bool isleader = act && leader == (int)lane;
    int id = -1;
    if (isleader && b > 0) {
      for (int j = 0; j < b; ++j)
        if ((unsigned)P.ckey[j] == key) {
          id = P.cid[j];
          break;
        }
    }
    const bool disc = isleader && id < 0;
    const unsigned dm = __ballot_sync(kFull, disc);
    if (disc) id = nkept + nnew + __popc(dm & lt);
    id = __shfl_sync(kFull, id, leader);
    if (act) P.cid[k] = (VId)id;
    if (disc) {
      const int r = id - nkept;
      if (r < C::NCAP) {
        const int p = P.cpos[k];
        const int s = P.fi[cb][p], e = P.fe[p];
        double ds, de;
        if constexpr (!C::MIXED) {
          ds = P.dist[s];
          de = P.dist[e];
        } else {  // the plain path's FP64 distances, needed only here
          ds = (P.vx[s] - px) * nx + (P.vy[s] - py) * ny + (P.vz[s] - pz) * nz;
          de = (P.vx[e] - px) * nx + (P.vy[e] - py) * ny + (P.vz[e] - pz) * nz;
        }
        const double t = clamp01(ds / (ds - de));
        const double ax = P.vx[s], ay = P.vy[s], az = P.vz[s];
        const double bx = P.vx[e], by = P.vy[e], bz = P.vz[e];
        const double ix = ax + t * (bx - ax);
        const double iy = ay + t * (by - ay);
        const double iz = az + t * (bz - az);
        if constexpr (kRegX) {
          rx = ix;
          ry = iy;
          rz = iz;
          rslot = r;
        } else {
          P.tx[r] = ix;
          P.ty[r] = iy;
          P.tz[r] = iz;
        }
        if (with_gen) {
          double dx = ix - gx;
          double dy = iy - gy;
          double dz = iz - gz;
          double d2 = dx * dx + dy * dy + dz * dz;
          r2 = fmax(r2, d2);
        }
      }
    }
    nnew += __popc(dm);
    __syncwarp();
  }
  cnt_add(P, kCntIntersections, (unsigned long long)nnew);
  const int nvn = nkept + nnew;
  if (nnew > C::NCAP || nvn > C::VCAP) return kClipOverflow;

  // 5. new vertex list: kept vertices compacted in place, then intersections
  double um = 0.0;
  for (int b = 0; b < nv; b += 32) {
    const int v = b + lane;
    unsigned o = C::VNONE;
    double x = 0.0, y = 0.0, z = 0.0;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    if (v < nv) {
      o = P.o2n[v];
      x = P.vx[v];
      y = P.vy[v];
      z = P.vz[v];
      if constexpr (C::MIXED) {
        fx = P.ux[v];
        fy = P.uy[v];
        fz = P.uz[v];
      }
    }
    __syncwarp();
    if (o != C::VNONE) {
      P.vx[o] = x;
      P.vy[o] = y;
      P.vz[o] = z;
      if constexpr (C::MIXED) {
        P.ux[o] = fx;
        P.uy[o] = fy;
        P.uz[o] = fz;
        um = fmax(um, fmax(fabs((double)fx), fmax(fabs((double)fy), fabs((double)fz))));
      }
    }
    __syncwarp();
  }
  auto place = [&](int r, double x, double y, double z) {
    P.vx[nkept + r] = x;
    P.vy[nkept + r] = y;
    P.vz[nkept + r] = z;
    if constexpr (C::MIXED) {
      const float fx = (float)(x - gx), fy = (float)(y - gy), fz = (float)(z - gz);
      P.ux[nkept + r] = fx;
      P.uy[nkept + r] = fy;
      P.uz[nkept + r] = fz;
      um = fmax(um, fmax(fabs((double)fx), fmax(fabs((double)fy), fabs((double)fz))));
    }
  };
  if constexpr (kRegX) {
    if (rslot >= 0) place(rslot, rx, ry, rz);
  } else {
    for (int r = lane; r < nnew; r += 32) place(r, P.tx[r], P.ty[r], P.tz[r]);
  }
  if constexpr (C::MIXED) S.umax = warp_max(um) * (1.0 + 0x1p-20);

  // 6. surviving faces (>= 3 entries, :454-467) and their new starts
  int nfk = 0, hk = 0;
  bool longface = false;
  for (int b = 0; b < nf; b += 32) {
    const int f = b + lane;
    int L = 0;
    if (f < nf) L = (int)P.E[P.fs[cb][f + 1]] - (int)P.E[P.fs[cb][f]];
    const bool kept = L >= 3;
    longface |= L > 255;  // the reference stores face sizes as u8
    const unsigned km = __ballot_sync(kFull, kept);
    const int Lk = kept ? L : 0;
    const int inc = warp_incl_scan(Lk);
    if (f < nf) {
      P.fnew[f] = kept ? (FId)(nfk + __popc(km & lt)) : (FId)C::FNONE;
      P.fns[f] = (typename C::Pos)(hk + inc - Lk);
      P.fdel[f] = (typename C::Del)(hk + inc - Lk - (int)P.E[P.fs[cb][f]]);
    }
    nfk += __popc(km);
    hk += __shfl_sync(kFull, inc, 31);
  }
  if (__any_sync(kFull, longface) || hk > C::HCAP) return kClipOverflow;
  __syncwarp();

  // 7. write the surviving faces' entries
  for (int p = lane; p < nh; p += 32) {
    const int f = P.pf[cb][p];
    const unsigned fw = P.fnew[f];
    if (fw != C::FNONE) {
      const VPair<VId> ve = P.pve[p];
      const unsigned os = ve.s, oe = ve.e;
      const bool si = os != C::VNONE, ei = oe != C::VNONE;
      const int o = (int)P.fdel[f] + (int)P.E[p];
      if (si) {
        P.fi[nb][o] = (VId)(ei ? oe : (unsigned)P.cid[P.cidx[p]]);
        P.pf[nb][o] = (FId)fw;
      } else if (ei) {
        P.fi[nb][o] = P.cid[P.cidx[p]];
        P.pf[nb][o] = (FId)fw;
        P.fi[nb][o + 1] = (VId)oe;
        P.pf[nb][o + 1] = (FId)fw;
      }
    }
  }
  //    and collect the lid segments.  In a face buffer two intersection
  //    entries are adjacent exactly when an in->out position is followed
  //    (after out->out positions) by an out->in one; the reference records
  //    (v, u) = (X of the out->in, X of the in->out), ordered by u's place in
  //    the buffer, i.e. by position -- the order of the crossing list
  int nseg = 0;
  for (int b = 0; b < ncross; b += 32) {
    const int kc = b + (int)lane;
    bool segsrc = false;
    int f = 0;
    if (kc < ncross) {
      const int p = P.cpos[kc];
      const VPair<VId> ve = P.pve[p];
      if (ve.s != C::VNONE && ve.e == C::VNONE) {
        f = P.pf[cb][p];
        segsrc = P.fnew[f] != C::FNONE;
      }
    }
    const unsigned sm = __ballot_sync(kFull, segsrc);
    if (segsrc) {
      const int k = nseg + __popc(sm & lt);
      if (k < C::SCAP) {
        // the out->in position that closes this in->out one is the next
        // crossing along the face (the positions between are out->out):
        // the next crossing in walk order if it lies in the same face, else
        // the face's first crossing
        int kn = kc + 1;
        if (kn >= ncross || (int)P.cpos[kn] >= (int)P.fs[cb][f + 1]) kn = P.fcr[f];
        P.sega[k] = P.cid[kn];
        P.segb[k] = P.cid[kc];
      }
    }
    nseg += __popc(sm);
  }
  for (int f = lane; f < nf; f += 32) {
    const unsigned fw = P.fnew[f];
    if (fw != C::FNONE) {
      P.fs[nb][fw] = P.fns[f];
      P.fn[nb][fw] = P.fn[cb][f];
    }
  }
  if (lane == 0) P.fs[nb][nfk] = (typename C::Pos)hk;
  if (nseg > C::SCAP) return kClipOverflow;

  // 8. lid (:470-495): lid_map (last writer wins) and the chain from the
  //    first segment, appended as the last face
  int nhn = hk, nfn = nfk;
  if (nseg > 0) {
    __syncwarp();
    for (int v = nkept + lane; v < nvn; v += 32) P.lidmap[v] = (VId)C::VNONE;
    __syncwarp();
    int len = 0, ovf = 0;
    // Common case: at most 32 segments, their starts distinct, their ends
    // distinct, every end the start of a segment.  The lid map is then a
    // permutation of the segments, and the chain from segment 0 (which the
    // serial walk below follows) is ranked by pointer jumping: the cycle is
    // cut before segment 0 and each segment's distance to the cut gives its
    // place in the lid face.
    bool fastlid = false;
    if (nseg <= 32) {
      const bool act = (int)lane < nseg;
      const unsigned a = act ? (unsigned)P.sega[lane] : (0xFFFF0000u | lane);
      const unsigned bend = act ? (unsigned)P.segb[lane] : (0xFFFE0000u | lane);
      const unsigned ma = __match_any_sync(kFull, a);
      const unsigned mb = __match_any_sync(kFull, bend);
      if (act) P.lidmap[a] = (VId)lane;
      __syncwarp();
      unsigned succ = lane;
      bool good = true;
      if (act) {
        succ = P.lidmap[bend];
        good = __popc(ma) == 1 && __popc(mb) == 1 && succ < (unsigned)nseg;
      }
      __syncwarp();
      if (__all_sync(kFull, good)) {
        fastlid = true;
        const int term = __ffs(__ballot_sync(kFull, act && succ == 0u)) - 1;
        int nxt = (act && (int)lane != term) ? (int)succ : (int)lane;
        int d = nxt != (int)lane ? 1 : 0;
        for (int span = 1; span < nseg; span <<= 1) {
          const int dn = __shfl_sync(kFull, d, nxt);
          const int nn = __shfl_sync(kFull, nxt, nxt);
          d += dn;
          nxt = nn;
        }
        const int d0 = __shfl_sync(kFull, d, 0);
        len = d0 + 1;
        if (hk + len > C::HCAP) ovf = 1;
        else if (act && nxt == term) P.fi[nb][hk + d0 - d] = (VId)a;
      } else {
        // restore the lid map's empty entries for the serial walk
        if (act) P.lidmap[a] = (VId)C::VNONE;
        __syncwarp();
      }
    }
    if (!fastlid) {
    for (int b = 0; b < nseg; b += 32) {
      const int k = b + lane;
      const bool act = k < nseg;
      const unsigned key = act ? (unsigned)P.sega[k] : (0xFFFF0000u | lane);
      const unsigned mm = __match_any_sync(kFull, key);
      const int last = 31 - __clz(mm);
      if (act && last == (int)lane) P.lidmap[key] = P.segb[k];
      __syncwarp();
    }
    if (lane == 0) {
      const unsigned start = P.sega[0];
      unsigned cur = P.segb[0];
      if (hk < C::HCAP) {
        P.fi[nb][hk] = (VId)start;
        len = 1;
        while (cur != start && len <= nseg) {
          if (hk + len >= C::HCAP) {
            ovf = 1;
            break;
          }
          P.fi[nb][hk + len] = (VId)cur;
          ++len;
          cur = P.lidmap[cur];
          if (cur == C::VNONE) break;
        }
      } else {
        ovf = 1;
      }
    }
    len = __shfl_sync(kFull, len, 0);
    ovf = __shfl_sync(kFull, ovf, 0);
    }
    if (ovf) return kClipOverflow;
    if (len >= 3) {
      if (nfk + 1 > C::FCAP || len > 255) return kClipOverflow;
      for (int q = lane; q < len; q += 32) P.pf[nb][hk + q] = (FId)nfk;
      if (lane == 0) {
        P.fs[nb][nfk] = (typename C::Pos)hk;
        P.fn[nb][nfk] = nbr;
        P.fs[nb][nfk + 1] = (typename C::Pos)(hk + len);
      }
      nhn = hk + len;
      nfn = nfk + 1;
    }
  }
  __syncwarp();
  S.nv = nvn;
  S.nf = nfn;
  S.nh = nhn;
  S.cb = nb;
  *r2out = with_gen ? warp_max(r2) : 0.0;
  return kClipMod;
}

// Whether clip_with_scratch with this lane's own plane (a different one per
// lane) would change the polytope: some vertex lies outside, d > 1e-9, with d
// computed as the clip computes it (:302-326).  Every lane walks every vertex
// in the same order (broadcast reads).
template <class C>
__device__ __forceinline__ bool plane_cuts(const WarpPoly<C>& P, const PolyState& S, double px, double py,
                                           double pz, double nx, double ny, double nz) {
  bool cut = false;
  for (int v = 0; v < S.nv; ++v) {
    const double d = (P.vx[v] - px) * nx + (P.vy[v] - py) * ny + (P.vz[v] - pz) * nz;
    cut |= d > kTol;
  }
  return cut;
}

template <class C>
__device__ __forceinline__ int poly_nverts(const WarpPoly<C>&, const PolyState& S) {
  return S.nv;
}

// in the walk's variant with batched plane tests (compute_cell<C, true>):
// with a run of TessDesc::noop_run clips that changed nothing and at least
// kNoopBatch candidates passing the radius tests, the candidates' planes are
// tested together.  The variant is a separate kernel: the test's code in the
// walk costs the common path registers (uniform input: 40.3 against 34.8 ms
// per 1 M cells with the test compiled in and never taken).
constexpr int kNoopBatch = 8;

// instrumented runs: the candidates of the bins the walk opens when it
// reaches entries (elo, ehi] of this chunk at radius^2 c4/4 -- every member
// but the cell's own generator (algo_3d_grid.rs:190-196)
template <class PolyT>
__device__ __forceinline__ void count_opened(PolyT& P, int elo, int ehi, bool valid, bool inr, bool own,
                                             double md2, double b2, uint32_t members, double c4) {
  const int l = (int)lane_id();
  const bool open = l > elo && l <= ehi && valid && inr && !(md2 > c4) && b2 <= c4;
  int c = open ? (int)members - (own ? 1 : 0) : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
  cnt_add(P, kCntCandidates, (unsigned long long)c);
}

// compute_cell (tessellation.rs:414-475) with Algorithm3DGrid::visit_neighbors
// (algo_3d_grid.rs:145-202) and the bisector visitor (tessellation.rs:446-471).
//
// The search order is consumed 32 entries at a time, one entry per lane
// (bin, exact bin lower bound, member range).  The members of the bins that
// can still open are flattened into one candidate list, 32 candidates per
// round, one per lane, loaded together.  Ballots against the CURRENT radius
// then pick, in order, exactly the candidates the reference clips with:
//  - the walk ends at the first entry past the bin being processed whose
//    min_d2 > 4R^2 (min_d2 ascends along the order; R only shrinks);
//  - a bin opens when its lower bound is <= 4R^2 at the moment the walk
//    reaches it -- for every bin past the last clipped candidate's, that is
//    the current R; the bin being processed already opened;
//  - a member is clipped with when dist^2 <= 4R^2 at its turn.
// Each clip may shrink R, and the ballots are re-evaluated after it.
template <class C, bool NOOP = false, class PolyT>
__device__ int compute_cell(const TessDesc& T, uint32_t i, PolyT& P, typename PolyT::State& S) {
  const unsigned lane = lane_id();
  const double gx = T.gen[3 * (size_t)i], gy = T.gen[3 * (size_t)i + 1], gz = T.gen[3 * (size_t)i + 2];
  double r2;
  poly_init_box(P, S, T.grid, gx, gy, gz);
  for (int w = 0; w < T.nwalls; ++w) {
    const Wall& W = T.walls[w];
    // one plane per generator, or a polyhedron's fixed planes in order
    const int np = W.kind == kWallPolyhedron ? W.np : 1;
    for (int k = 0; k < np; ++k) {
      double p[3], n[3];
      bool emit;
      if (W.kind == kWallPolyhedron) {
        const double* pl = T.planes + 6 * (W.p0 + k);
        p[0] = pl[0];
        p[1] = pl[1];
        p[2] = pl[2];
        n[0] = pl[3];
        n[1] = pl[4];
        n[2] = pl[5];
        emit = true;
      } else {
        emit = wall_plane(W, gx, gy, gz, p, n);
      }
      if (emit) {
        const int r = warp_clip(P, S, p[0], p[1], p[2], n[0], n[1], n[2], W.id, false, gx, gy, gz, &r2);
        if (r == kClipOverflow) return kCellOverflow;
      }
    }
    if (state_empty(S)) return kCellOk;
  }
  double cur = poly_max_radius_sq(P, S, gx, gy, gz);

  const Grid& G = T.grid;
  const uint32_t bin = T.bin_of[i];
  const uint32_t nxy = (uint32_t)G.n[0] * (uint32_t)G.n[1];
  const int iz = (int)(bin / nxy);
  const uint32_t rem = bin % nxy;
  const int iy = (int)(rem / (uint32_t)G.n[0]);
  const int ix = (int)(rem % (uint32_t)G.n[0]);
  const double rx = (gx - G.bmin[0]) * G.scale[0] - (double)ix;
  const double ry = (gy - G.bmin[1]) * G.scale[1] - (double)iy;
  const double rz = (gz - G.bmin[2]) * G.scale[2] - (double)iz;

  bool done = false;
  [[maybe_unused]] int nnoop = 0;  // clips in a row that changed nothing (NOOP)
  for (int base = 0; base < T.norder && !done; base += 32) {
    // ---- this lane's search-order entry ----
    const int k = base + (int)lane;
    const bool valid = k < T.norder;
    double md2 = 0.0, b2 = 0.0;
    bool inr = false, own = false;
    uint32_t bs = 0, be = 0;
    if (valid) {
      const Offset o = T.order[k];
      md2 = o.min_d2;
      own = o.dx == 0 && o.dy == 0 && o.dz == 0;
      const int bx = ix + o.dx, by = iy + o.dy, bz = iz + o.dz;
      inr = bx >= 0 && bx < G.n[0] && by >= 0 && by < G.n[1] && bz >= 0 && bz < G.n[2];
      if (inr) {
        const uint32_t bb = (uint32_t)bx + (uint32_t)by * (uint32_t)G.n[0] + (uint32_t)bz * nxy;
        // on sparse grids an empty bin is known from its occupancy bit (an
        // L2-resident map) without reading the bin table; an empty bin opens
        // nothing, so its lower bound is needed only for occupied bins
        if (!T.occ || ((__ldg(&T.occ[bb >> 5]) >> (bb & 31u)) & 1u)) {
          bs = T.bin_start[bb];
          be = T.bin_start[bb + 1];
          const double ddx = o.dx > 0 ? ((double)o.dx - rx) * G.cs[0]
                                      : (o.dx < 0 ? ((double)(-(o.dx + 1)) + rx) * G.cs[0] : 0.0);
          const double ddy = o.dy > 0 ? ((double)o.dy - ry) * G.cs[1]
                                      : (o.dy < 0 ? ((double)(-(o.dy + 1)) + ry) * G.cs[1] : 0.0);
          const double ddz = o.dz > 0 ? ((double)o.dz - rz) * G.cs[2]
                                      : (o.dz < 0 ? ((double)(-(o.dz + 1)) + rz) * G.cs[2] : 0.0);
          const double bdx = fmax(ddx, 0.0), bdy = fmax(ddy, 0.0), bdz = fmax(ddz, 0.0);
          b2 = bdx * bdx + bdy * bdy + bdz * bdz;
        }
      }
    }
    const int nvalid = min(32, T.norder - base);
    // bins that can still open (R only shrinks), flattened: members of entry
    // e are candidates [start, start + cnt)
    const bool pot = valid && inr && be > bs && !(md2 > 4.0 * cur) && b2 <= 4.0 * cur;
    if (!__any_sync(kFull, pot)) {
      // no bin of this chunk can open (sparse regions, fine grids): only
      // the end of the walk is decided here
      const unsigned brk = __ballot_sync(kFull, valid && md2 > 4.0 * cur);
      const int fbe = brk ? __ffs(brk) - 1 : 32;
      if constexpr (C::COUNT) cnt_add(P, kCntOffsets, (unsigned long long)(fbe < 32 ? fbe + 1 : nvalid));
      if (fbe < 32) done = true;
      continue;
    }
    const int cnt = pot ? (int)(be - bs) : 0;
    const int incl = warp_incl_scan(cnt);
    const int start = incl - cnt;
    const int total = __shfl_sync(kFull, incl, 31);
    int ecur = -1;  // entry of the bin being processed (opened)
    int pos = 0;    // next candidate to consider
    int fb = 32;    // entry that ends the walk (32: none in this chunk)
    for (int r0 = 0;; r0 += 32) {
      if (r0 < total) {
        const int lo = max(start, r0), hi = min(start + cnt, r0 + 32);
        for (int q = lo; q < hi; ++q) P.cand_e[q - r0] = (uint8_t)lane;
      }
      __syncwarp();
      const int idx = r0 + (int)lane;
      const bool have = idx < total;
      const int ce = have ? (int)P.cand_e[lane] : 0;
      __syncwarp();
      const uint32_t cbs = __shfl_sync(kFull, bs, ce);
      const int cst = __shfl_sync(kFull, start, ce);
      const double cb2 = __shfl_sync(kFull, b2, ce);
      SortedGen sg = {0.0, 0.0, 0.0, -1};
      if (have) sg = T.sorted[cbs + (uint32_t)(idx - cst)];
      const bool cand = have && sg.id != (long long)i;
      const double d0 = sg.x - gx, d1 = sg.y - gy, d2 = sg.z - gz;
      const double dist_sq = d0 * d0 + d1 * d1 + d2 * d2;
      while (true) {
        const double c4 = 4.0 * cur;
        const unsigned later = ecur < 0 ? kFull : (ecur >= 31 ? 0u : ~((2u << ecur) - 1u));
        const unsigned brk = __ballot_sync(kFull, valid && md2 > c4) & later;
        fb = brk ? __ffs(brk) - 1 : 32;
        const bool ok = cand && idx >= pos && ce < fb && !(dist_sq > c4) && (ce == ecur || cb2 <= c4);
        const unsigned pass = __ballot_sync(kFull, ok);
        if (!pass) break;
        if constexpr (NOOP) {
          if (T.noop_run > 0 && nnoop >= T.noop_run && __popc(pass) >= kNoopBatch) {
            // in a run of clips that changed nothing (a cell whose radius still
            // reaches far, e.g. at the edge of a populated region), the passing
            // candidates' planes are tested together, one per lane, and those
            // before the first plane that cuts are passed over: clipping with
            // them would change neither the polytope nor R, and the candidates
            // that pass do not change either (the reference's sequence, bit for bit)
            const bool cuts =
                plane_cuts(P, S, gx + d0 * 0.5, gy + d1 * 0.5, gz + d2 * 0.5, d0, d1, d2);
            const unsigned cm = __ballot_sync(kFull, cuts) & pass;
            const unsigned skip = cm ? pass & ((1u << (__ffs(cm) - 1)) - 1u) : pass;
            if (skip) {
              const int jl = 31 - __clz(skip);
              const int el = __shfl_sync(kFull, ce, jl);
              if constexpr (C::COUNT) {
                count_opened(P, ecur, el, valid, inr, own, md2, b2, be - bs, c4);
                cnt_add(P, kCntClips, (unsigned long long)__popc(skip));
                cnt_add(P, kCntClassified, (unsigned long long)__popc(skip) * (unsigned long long)poly_nverts(P, S));
              }
              ecur = el;
              pos = r0 + jl + 1;
              continue;
            }
          }
        }
        const int j = __ffs(pass) - 1;
        const int ej = __shfl_sync(kFull, ce, j);
        if constexpr (C::COUNT) count_opened(P, ecur, ej, valid, inr, own, md2, b2, be - bs, c4);
        const int jid = (int)__shfl_sync(kFull, sg.id, j);
        const double e0 = __shfl_sync(kFull, d0, j);
        const double e1 = __shfl_sync(kFull, d1, j);
        const double e2 = __shfl_sync(kFull, d2, j);
        const double mx = gx + e0 * 0.5, my = gy + e1 * 0.5, mz = gz + e2 * 0.5;
        const int r = warp_clip(P, S, mx, my, mz, e0, e1, e2, jid, true, gx, gy, gz, &r2);
        if (r == kClipOverflow) return kCellOverflow;
        if (r == kClipMod) cur = r2;
        else if (r == kClipEmpty) cur = 0.0;
        if constexpr (NOOP) nnoop = r == kClipNoop ? nnoop + 1 : 0;
        ecur = ej;
        pos = r0 + j + 1;
      }
      if (r0 + 32 >= total) break;
      // the next round starts at an entry the walk no longer reaches
      const unsigned nxt = __ballot_sync(kFull, cnt > 0 && start <= r0 + 32);
      if (fb < 32 && 31 - __clz(nxt) >= fb) break;
    }
    if constexpr (C::COUNT) {
      count_opened(P, ecur, fb < 32 ? fb - 1 : 31, valid, inr, own, md2, b2, be - bs, 4.0 * cur);
      cnt_add(P, kCntOffsets, (unsigned long long)(fb < 32 ? fb + 1 : nvalid));
    }
    if (fb < 32) done = true;
  }
  if (!done && !T.order_complete && !(T.order_bound > 4.0 * cur)) return kCellTable;
  return kCellOk;
}

// volume + centroid (cell_3d_faces.rs:106-205) summed in the reference's
// order, and face_area (:207-254) per face; writes the cell's outputs.
template <class C>
__device__ void finalize_cell(const TessDesc& T, uint32_t i, WarpPoly<C>& P, const PolyState& S) {
  const unsigned lane = lane_id();
  const int cb = S.cb, nb = cb ^ 1;
  const int nf = S.nf;
  // triangle prefix over faces; triangle -> face map in the spare buffer
  int ntri = 0;
  for (int b = 0; b < nf; b += 32) {
    const int f = b + lane;
    int t = 0;
    if (f < nf) {
      const int c = (int)P.fs[cb][f + 1] - (int)P.fs[cb][f];
      t = c >= 3 ? c - 2 : 0;
    }
    const int inc = warp_incl_scan(t);
    if (f < nf) P.E[f] = (typename C::Pos)(ntri + inc - t);
    ntri += __shfl_sync(kFull, inc, 31);
  }
  __syncwarp();
  for (int f = lane; f < nf; f += 32) {
    const int c = (int)P.fs[cb][f + 1] - (int)P.fs[cb][f];
    for (int j = 0; j < c - 2; ++j) P.pf[nb][P.E[f] + j] = (typename C::FId)f;
  }
  __syncwarp();
  double av = 0.0, ax = 0.0, ay = 0.0, az = 0.0;
  for (int b = 0; b < ntri; b += 32) {
    const int t = b + lane;
    double det = 0.0, dtx = 0.0, dty = 0.0, dtz = 0.0;
    if (t < ntri) {
      const int f = P.pf[nb][t];
      const int base = P.fs[cb][f];
      const int j = t - (int)P.E[f] + 1;
      const int i0 = P.fi[cb][base], i1 = P.fi[cb][base + j], i2 = P.fi[cb][base + j + 1];
      const double v0x = P.vx[i0], v0y = P.vy[i0], v0z = P.vz[i0];
      const double v1x = P.vx[i1], v1y = P.vy[i1], v1z = P.vz[i1];
      const double v2x = P.vx[i2], v2y = P.vy[i2], v2z = P.vz[i2];
      const double crx = v1y * v2z - v1z * v2y;
      const double cry = v1z * v2x - v1x * v2z;
      const double crz = v1x * v2y - v1y * v2x;
      det = v0x * crx + v0y * cry + v0z * crz;
      dtx = det * (v0x + v1x + v2x);
      dty = det * (v0y + v1y + v2y);
      dtz = det * (v0z + v1z + v2z);
    }
    const int cntt = min(32, ntri - b);
    for (int j = 0; j < cntt; ++j) {
      av += __shfl_sync(kFull, det, j);
      ax += __shfl_sync(kFull, dtx, j);
      ay += __shfl_sync(kFull, dty, j);
      az += __shfl_sync(kFull, dtz, j);
    }
  }
  cnt_add(P, kCntTriangles, (unsigned long long)ntri);
  const int fout = T.fout;
  int32_t* fnb_out = nullptr;
  double* far_out = nullptr;
  if (nf <= fout) {
    fnb_out = T.fnb + (size_t)i * fout;
    far_out = T.farea + (size_t)i * fout;
  } else if (T.pool_cursor) {
    unsigned long long off = 0;
    if (lane == 0) off = atomicAdd(T.pool_cursor, (unsigned long long)nf);
    off = __shfl_sync(kFull, off, 0);
    if ((long long)(off + nf) <= T.pool_cap) {
      fnb_out = T.pool_fnb + off;
      far_out = T.pool_farea + off;
      if (lane == 0) T.pool_off[i] = (long long)off;
    }
  }
  for (int f = lane; f < nf; f += 32) {
    const int base = P.fs[cb][f];
    const int c = (int)P.fs[cb][f + 1] - base;
    double area = 0.0;
    if (c >= 3) {
      const int p0 = P.fi[cb][base];
      const double p0x = P.vx[p0], p0y = P.vy[p0], p0z = P.vz[p0];
      for (int j = 1; j < c - 1; ++j) {
        const int p1 = P.fi[cb][base + j], p2 = P.fi[cb][base + j + 1];
        const double v1x = P.vx[p1] - p0x, v1y = P.vy[p1] - p0y, v1z = P.vz[p1] - p0z;
        const double v2x = P.vx[p2] - p0x, v2y = P.vy[p2] - p0y, v2z = P.vz[p2] - p0z;
        const double crx = v1y * v2z - v1z * v2y;
        const double cry = v1z * v2x - v1x * v2z;
        const double crz = v1x * v2y - v1y * v2x;
        area += 0.5 * sqrt(crx * crx + cry * cry + crz * crz);
      }
    }
    if (fnb_out) {
      fnb_out[f] = P.fn[cb][f];
      far_out[f] = area;
    }
  }
  if (lane == 0) {
    T.vol[i] = fabs(av / 6.0);
    if (fabs(av) < 1e-9) {
      T.cen[3 * (size_t)i] = 0.0;
      T.cen[3 * (size_t)i + 1] = 0.0;
      T.cen[3 * (size_t)i + 2] = 0.0;
    } else {
      const double factor = 1.0 / (4.0 * av);
      T.cen[3 * (size_t)i] = ax * factor;
      T.cen[3 * (size_t)i + 1] = ay * factor;
      T.cen[3 * (size_t)i + 2] = az * factor;
    }
    T.nfaces[i] = (fnb_out || nf == 0) ? nf : -1;
    T.nverts[i] = S.nv;
    T.status[i] = (fnb_out || nf == 0) ? kCellOk : kCellHardFail;
  }
}

template <class C>
__device__ void export_cell(const WorkList& W, const WarpPoly<C>& P, const PolyState& S) {
  const unsigned lane = lane_id();
  if (lane == 0) {
    W.ex_sizes[0] = S.nv;
    W.ex_sizes[1] = S.nf;
    W.ex_sizes[2] = S.nh;
  }
  if (S.nv <= W.ex_cap_v)
    for (int v = lane; v < S.nv; v += 32) {
      W.ex_verts[3 * v] = P.vx[v];
      W.ex_verts[3 * v + 1] = P.vy[v];
      W.ex_verts[3 * v + 2] = P.vz[v];
    }
  if (S.nf <= W.ex_cap_f)
    for (int f = lane; f < S.nf; f += 32) {
      W.ex_fc[f] = (uint32_t)(P.fs[S.cb][f + 1] - P.fs[S.cb][f]);
      W.ex_fn[f] = P.fn[S.cb][f];
    }
  if (S.nh <= W.ex_cap_h)
    for (int h = lane; h < S.nh; h += 32) W.ex_fi[h] = P.fi[S.cb][h];
}

// Persistent warps pull cells from the work list and build them.
template <class C, bool NOOP = false, class PolyT>
__device__ void clip_worker(const TessDesc& T, const WorkList& W, PolyT& P) {
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
    const uint32_t cell = W.items ? W.items[idx] : (uint32_t)T.sorted[idx].id;
    typename PolyT::State S;
    const int st = compute_cell<C, NOOP>(T, cell, P, S);
    if (st == kCellOk) {
      finalize_cell<C>(T, cell, P, S);
      if constexpr (PolyT::kExport) {
        if (W.ex_verts) export_cell<C>(W, P, S);
      }
    } else if (lane == 0) {
      T.status[cell] = (uint8_t)st;
      if (st == kCellOverflow && W.ovf_list) W.ovf_list[atomicAdd(W.ovf_count, 1u)] = cell;
      if (st == kCellTable && W.tab_list) W.tab_list[atomicAdd(W.tab_count, 1u)] = cell;
    }
    __syncwarp();
  }
  __syncwarp();
  if constexpr (C::COUNT) {
    if (lane < kNumCounters && W.counters) atomicAdd(&W.counters[lane], P.cnt[lane]);
  }
}

// Batched mode: one work item per cell of many tessellations.  Items are
// global positions in the concatenated bin-ordered generator array;
// tess_off[t] is tessellation t's first position (tess_off[ntess] = total).
__device__ __forceinline__ int find_tess(const uint32_t* tess_off, int ntess, uint32_t item) {
  int lo = 0, hi = ntess;  // largest t with tess_off[t] <= item
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (tess_off[mid] <= item) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <class C, class PolyT>
__device__ void clip_worker_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess,
                                    const WorkList& W, PolyT& P) {
  const unsigned lane = lane_id();
  if constexpr (C::COUNT) {
    if (lane < kNumCounters) P.cnt[lane] = 0;
  }
  const uint32_t nitems = W.nitems_dev ? *W.nitems_dev : W.nitems;
  __syncwarp();
  while (true) {
    unsigned idx = 0;
    if (lane == 0) idx = atomicAdd(W.cursor, 1u);
    idx = __shfl_sync(kFull, idx, 0);
    if (idx >= nitems) break;
    const uint32_t item = W.items ? W.items[idx] : idx;
    const int t = find_tess(tess_off, ntess, item);
    const TessDesc& T = descs[t];
    const uint32_t cell = (uint32_t)T.sorted[item].id;
    typename PolyT::State S;
    const int st = compute_cell<C>(T, cell, P, S);
    if (st == kCellOk) {
      finalize_cell<C>(T, cell, P, S);
    } else if (lane == 0) {
      T.status[cell] = (uint8_t)st;
      if (st == kCellOverflow && W.ovf_list) W.ovf_list[atomicAdd(W.ovf_count, 1u)] = item;
      if (st == kCellTable) {
        if (W.tab_list) W.tab_list[atomicAdd(W.tab_count, 1u)] = item;
        if (W.tess_flags) atomicOr(&W.tess_flags[t], 1u);
      }
    }
    __syncwarp();
  }
  __syncwarp();
  if constexpr (C::COUNT) {
    if (lane < kNumCounters && W.counters) atomicAdd(&W.counters[lane], P.cnt[lane]);
  }
}

// The kernels: persistent warps over a work list; the fast path keeps each
// warp's polytope in shared memory, the large-capacity pass in a slice of a
// global scratch buffer.
constexpr int kFastWarpsPerBlock = 4;

// MINB: blocks per SM the register budget must admit (shared memory sets it);
// NOOP: the walk's variant with batched plane tests (compute_cell)
template <class C, int WPB, int MINB, bool NOOP = false>
__global__ void __launch_bounds__(WPB * 32, MINB) k_clip_fast(const TessDesc T, const WorkList W) {
  extern __shared__ __align__(16) unsigned char smem[];
  WarpPoly<C>* polys = reinterpret_cast<WarpPoly<C>*>(smem);
  clip_worker<C, NOOP>(T, W, polys[threadIdx.x >> 5]);
}

template <class C, bool NOOP = false>
__global__ void __launch_bounds__(128) k_clip_big(const TessDesc T, const WorkList W, WarpPoly<C>* scratch) {
  const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  clip_worker<C, NOOP>(T, W, scratch[gw]);
}

template <class C, int WPB, int MINB>
__global__ void __launch_bounds__(WPB * 32, MINB)
    k_clip_fast_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess, const WorkList W) {
  extern __shared__ __align__(16) unsigned char smem[];
  WarpPoly<C>* polys = reinterpret_cast<WarpPoly<C>*>(smem);
  clip_worker_batched<C>(descs, tess_off, ntess, W, polys[threadIdx.x >> 5]);
}

template <class C>
__global__ void __launch_bounds__(128)
    k_clip_big_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess, const WorkList W,
                       WarpPoly<C>* scratch) {
  const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  clip_worker_batched<C>(descs, tess_off, ntess, W, scratch[gw]);
}

}  // namespace vd
