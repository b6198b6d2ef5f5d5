// vd_clip_block.cuh -- the huge tier: one thread block per cell.
//
// A cell adjacent to thousands of others (the centre of generators on a
// sphere has N-1 faces) is clipped thousands of times while its polytope holds
// tens of thousands of vertices and face entries.  One warp (warp_clip) walks
// such a polytope 32 elements at a time through chains of dependent loads; here
// the NW warps of a block split every pass over vertices, faces and face
// positions into NW contiguous ranges.  Each prefix (vertex renumbering,
// crossing numbers, emitted entries, surviving faces, lid segments) is computed
// in two passes -- per-range totals, a scan of the NW totals, then the writes --
// so every element gets exactly the index warp_clip gives it and the output is
// the same polytope, bit for bit.  The short serial steps (the intersection
// vertices' first-occurrence numbering, the lid chain) run on warp 0 as in
// warp_clip.  The walk over candidates runs redundantly in every warp (each
// reads the same data and makes the same decisions) with a staging row per
// warp, and every warp enters each block_clip together.
#pragma once
#include "vd_clip.cuh"

namespace vd {

template <int NW>
struct BlockShared {
  int a[NW], b[NW], c[NW];     // per-range totals of a pass
  int val[8];                  // block-wide results
  double r2[NW];
  uint8_t cand[NW][32];        // the walk's candidate staging, a row per warp
  unsigned idx;
};

// warp w's contiguous share [lo, hi) of [0, n), whole chunks of 32
template <int NW>
__device__ __forceinline__ void block_range(int n, int w, int* lo, int* hi) {
  const int chunks = (n + 31) >> 5;
  const int per = (chunks + NW - 1) / NW;
  *lo = min(n, w * per * 32);
  *hi = min(n, (w + 1) * per * 32);
}

// every warp reads the NW range totals after the barrier that follows their
// writes and derives its own prefixes: exclusive sums of a[] and b[] before
// range w, the running maximum of c[] before it (-1 for none), and the
// totals (sums of a[] and b[], maximum of c[]) -- no second barrier.  The
// totals are rewritten only after the barrier that ends the pass using them.
template <int NW>
__device__ __forceinline__ void range_prefix(const BlockShared<NW>& B, int w, int* pa, int* pb, int* pc, int* ta,
                                             int* tb, int* tc) {
  static_assert(NW <= 32, "one range total per lane");
  const unsigned lane = lane_id();
  const bool in = (int)lane < NW;
  const int a = in ? B.a[lane] : 0, b = in ? B.b[lane] : 0, c = in ? B.c[lane] : -1;
  const int sa = warp_incl_scan(a), sb = warp_incl_scan(b);
  int mc = c;
  for (int d = 1; d < 32; d <<= 1) {
    const int o = __shfl_up_sync(kFull, mc, d);
    if ((int)lane >= d) mc = max(mc, o);
  }
  const int mprev = __shfl_up_sync(kFull, mc, 1);
  *pa = __shfl_sync(kFull, sa - a, w);
  *pb = __shfl_sync(kFull, sb - b, w);
  *pc = __shfl_sync(kFull, lane == 0 ? -1 : mprev, w);
  *ta = __shfl_sync(kFull, sa, 31);
  *tb = __shfl_sync(kFull, sb, 31);
  *tc = __shfl_sync(kFull, mc, 31);
}

// clip_with_scratch (cell_3d_faces.rs:288-503) by the whole block; every
// thread calls it with the same arguments and gets the same result.
template <class C, int NW>
__device__ int block_clip(WarpPoly<C>& P, BlockShared<NW>& B, PolyState& S, double px, double py,
                          double pz, double nx, double ny, double nz, int nbr, bool with_gen, double gx, double gy,
                          double gz, double* r2out) {
  static_assert(!C::MIXED && !C::COUNT, "the block clip is the plain FP64 path without counters");
  using VId = typename C::VId;
  using FId = typename C::FId;
  const unsigned lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  const int w = (int)(threadIdx.x >> 5);
  const int nt = NW * 32;
  const int tid = (int)threadIdx.x;
  const int nv = S.nv, nf = S.nf, nh = S.nh, cb = S.cb, nb = cb ^ 1;

  // 1. signed distances and the 3-band flags (:302-326); the kept vertices'
  //    squared distance from the generator (the clip's max radius)
  bool out = false, sin = false;
  double r2 = 0.0;
  for (int v = tid; v < nv; v += nt) {
    const double vx = P.vx[v], vy = P.vy[v], vz = P.vz[v];
    const double d = (vx - px) * nx + (vy - py) * ny + (vz - pz) * nz;
    P.dist[v] = d;
    P.o2n[v] = d > kTol ? (VId)C::VNONE : (VId)0;
    out |= d > kTol;
    sin |= d < -kTol;
    if (!(d > kTol) && with_gen) {
      double dx = vx - gx;
      double dy = vy - gy;
      double dz = vz - gz;
      double d2 = dx * dx + dy * dy + dz * dz;
      r2 = fmax(r2, d2);
    }
  }
  const bool any_out = __syncthreads_or(out) != 0;
  const bool any_sin = __syncthreads_or(sin) != 0;
  if (!any_out) {
    *r2out = 0.0;
    return kClipNoop;
  }
  if (!any_sin) {
    S.nv = S.nf = S.nh = 0;
    *r2out = 0.0;
    return kClipEmpty;
  }

  // 2. keep the inside vertices in order (:344-362)
  int lo, hi;
  block_range<NW>(nv, w, &lo, &hi);
  {
    int cnt = 0, first = nv;
    for (int b = lo; b < hi; b += 32) {
      const int v = b + lane;
      const unsigned km = __ballot_sync(kFull, v < hi && P.o2n[v] != C::VNONE);
      cnt += __popc(km);
      const unsigned rm = ~km & (hi - b >= 32 ? kFull : ((1u << (hi - b)) - 1u));
      if (rm && first == nv) first = b + __ffs(rm) - 1;
    }
    if (lane == 0) {
      B.a[w] = cnt;
      B.c[w] = first;
    }
  }
  __syncthreads();
  int nkept, run0, vfirst;
  {
    const bool in = (int)lane < NW;
    const int a = in ? B.a[lane] : 0;
    const int sa = warp_incl_scan(a);
    run0 = __shfl_sync(kFull, sa - a, w);
    nkept = __shfl_sync(kFull, sa, 31);
    vfirst = __reduce_min_sync(kFull, in ? B.c[lane] : nv);
  }
  {
    int run = run0;
    for (int b = lo; b < hi; b += 32) {
      const int v = b + lane;
      const bool k = v < hi && P.o2n[v] != C::VNONE;
      const unsigned m = __ballot_sync(kFull, k);
      if (v < hi) P.o2n[v] = k ? (VId)(run + __popc(m & lt)) : (VId)C::VNONE;
      run += __popc(m);
    }
  }
  __syncthreads();

  // 3. the face walk (:369-452): end vertices, crossings in walk order, the
  //    emitted-entry prefix E, each face's first crossing.  The first pass
  //    follows each position's chain of loads (face, its bounds, the edge's
  //    ends, their new ids) and keeps the end vertex and the new ids; the
  //    second reads those back and follows the chain again only at crossings.
  block_range<NW>(nh, w, &lo, &hi);
  {
    int ncr = 0, emit = 0, lastc = -1;
    for (int b = lo; b < hi; b += 32) {
      const int p = b + lane;
      bool cr = false, si = false, ei = false;
      if (p < hi) {
        const int f = P.pf[cb][p];
        const int f0 = P.fs[cb][f];
        const unsigned s = P.fi[cb][p];
        const unsigned e = P.fi[cb][(p + 1 == (int)P.fs[cb][f + 1]) ? f0 : p + 1];
        const VId os = P.o2n[s], oe = P.o2n[e];
        si = os != C::VNONE;
        ei = oe != C::VNONE;
        P.fe[p] = (VId)e;
        P.pve[p] = VPair<VId>{os, oe};
        cr = si != ei;
      }
      const unsigned m = __ballot_sync(kFull, cr);
      ncr += __popc(m);
      if (m) lastc = b + 31 - __clz(m);
      emit += __popc(__ballot_sync(kFull, si)) + 2 * __popc(__ballot_sync(kFull, !si && ei));
    }
    if (lane == 0) {
      B.a[w] = ncr;
      B.b[w] = emit;
      B.c[w] = lastc;
    }
  }
  __syncthreads();
  int ncross, emitted;
  {
    int nc, run, lastcross, unused;
    range_prefix<NW>(B, w, &nc, &run, &lastcross, &ncross, &emitted, &unused);
    for (int b = lo; b < hi; b += 32) {
      const int p = b + lane;
      bool cr = false, si = false, ei = false;
      if (p < hi) {
        const VPair<VId> ve = P.pve[p];
        si = ve.s != C::VNONE;
        ei = ve.e != C::VNONE;
        cr = si != ei;
      }
      const unsigned m = __ballot_sync(kFull, cr);
      if (cr) {
        const int k = nc + __popc(m & lt);
        const unsigned before = m & lt;
        const int prevp = before ? b + 31 - __clz(before) : lastcross;
        if (k < C::CCAP) {
          const int f = P.pf[cb][p];
          const int f0 = P.fs[cb][f];
          const unsigned s = P.fi[cb][p];
          const unsigned e = P.fe[p];
          P.cpos[k] = (typename C::Pos)p;
          P.ckey[k] = (typename C::Key)(s < e ? (s << C::KSHIFT | e) : (e << C::KSHIFT | s));
          P.cidx[p] = (typename C::CId)k;
          if (prevp < f0) P.fcr[f] = (typename C::CId)k;
        }
      }
      if (m) lastcross = b + 31 - __clz(m);
      nc += __popc(m);
      const unsigned m1 = __ballot_sync(kFull, si);
      const unsigned m2 = __ballot_sync(kFull, !si && ei);
      if (p < hi) P.E[p] = (typename C::Pos)(run + __popc(m1 & lt) + 2 * __popc(m2 & lt));
      run += __popc(m1) + 2 * __popc(m2);
    }
    if (tid == 0) P.E[nh] = (typename C::Pos)emitted;
  }
  __syncthreads();
  if (ncross > C::CCAP) return kClipOverflow;

  // 4. intersection vertices (warp 0): the first occurrence of an edge key
  //    creates the vertex, numbered in discovery order; repeats reuse it
  if (w == 0) {
    int nnew = 0;
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
          const double ds = P.dist[s], de = P.dist[e];
          const double t = clamp01(ds / (ds - de));
          const double ax = P.vx[s], ay = P.vy[s], az = P.vz[s];
          const double bx = P.vx[e], by = P.vy[e], bz = P.vz[e];
          const double ix = ax + t * (bx - ax);
          const double iy = ay + t * (by - ay);
          const double iz = az + t * (bz - az);
          P.tx[r] = ix;
          P.ty[r] = iy;
          P.tz[r] = iz;
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
    if (lane == 0) B.val[3] = nnew;
  }
  __syncthreads();
  const int nnew = B.val[3];
  const int nvn = nkept + nnew;
  if (nnew > C::NCAP || nvn > C::VCAP) return kClipOverflow;

  // 5. new vertex list: kept vertices compacted in place, then intersections.
  //    Vertices below the first removed one keep their index.  A kept vertex
  //    only moves down (o2n[v] <= v), so in rounds of consecutive vertices,
  //    read into registers before a barrier and written after it, no write
  //    reaches a vertex that is still to be read.
  {
    constexpr int K = 1;
    const int v0 = vfirst;
    for (int base = v0; base < nv; base += K * nt) {
      double bx[K], by[K], bz[K];
      int bo[K];
#pragma unroll
      for (int j = 0; j < K; ++j) {
        const int v = base + j * nt + tid;
        bo[j] = -1;
        if (v < nv) {
          const unsigned o = P.o2n[v];
          if (o != C::VNONE) {
            bo[j] = (int)o;
            bx[j] = P.vx[v];
            by[j] = P.vy[v];
            bz[j] = P.vz[v];
          }
        }
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < K; ++j) {
        if (bo[j] >= 0) {
          P.vx[bo[j]] = bx[j];
          P.vy[bo[j]] = by[j];
          P.vz[bo[j]] = bz[j];
        }
      }
    }
  }
  // (positions >= nkept were last read before the final round's barrier)
  for (int r = tid; r < nnew; r += nt) {
    P.vx[nkept + r] = P.tx[r];
    P.vy[nkept + r] = P.ty[r];
    P.vz[nkept + r] = P.tz[r];
  }

  // 6. surviving faces (>= 3 entries, :454-467) and their new starts
  block_range<NW>(nf, w, &lo, &hi);
  {
    int kept = 0, sum = 0, longf = 0;
    for (int b = lo; b < hi; b += 32) {
      const int f = b + lane;
      int L = 0;
      if (f < hi) L = (int)P.E[P.fs[cb][f + 1]] - (int)P.E[P.fs[cb][f]];
      const bool k = L >= 3;
      longf |= __any_sync(kFull, L > 255) ? 1 : 0;
      kept += __popc(__ballot_sync(kFull, k));
      sum += __shfl_sync(kFull, warp_incl_scan(k ? L : 0), 31);
    }
    if (lane == 0) {
      B.a[w] = kept;
      B.b[w] = sum;
      B.c[w] = longf;
    }
  }
  __syncthreads();
  int nfk, hk, lmax;
  int nfr, hr;
  {
    int unused;
    range_prefix<NW>(B, w, &nfr, &hr, &unused, &nfk, &hk, &lmax);
  }
  const bool longface = lmax > 0;
  {
    for (int b = lo; b < hi; b += 32) {
      const int f = b + lane;
      int L = 0;
      if (f < hi) L = (int)P.E[P.fs[cb][f + 1]] - (int)P.E[P.fs[cb][f]];
      const bool kept = L >= 3;
      const unsigned km = __ballot_sync(kFull, kept);
      const int Lk = kept ? L : 0;
      const int inc = warp_incl_scan(Lk);
      if (f < hi) {
        P.fnew[f] = kept ? (FId)(nfr + __popc(km & lt)) : (FId)C::FNONE;
        P.fns[f] = (typename C::Pos)(hr + inc - Lk);
        P.fdel[f] = (typename C::Del)(hr + inc - Lk - (int)P.E[P.fs[cb][f]]);
      }
      nfr += __popc(km);
      hr += __shfl_sync(kFull, inc, 31);
    }
  }
  __syncthreads();
  if (longface || hk > C::HCAP) return kClipOverflow;

  // 7. the surviving faces' entries (every thread), and the lid segments
  //    (v, u) ordered by the position of their in->out crossing: the crossing
  //    list is in position order, so warp 0 takes them from it
  for (int p = tid; p < nh; p += nt) {
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
  if (w == 0) {
    int k0 = 0;
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
        const int k = k0 + __popc(sm & lt);
        if (k < C::SCAP) {
          int kn = kc + 1;
          if (kn >= ncross || (int)P.cpos[kn] >= (int)P.fs[cb][f + 1]) kn = P.fcr[f];
          P.sega[k] = P.cid[kn];
          P.segb[k] = P.cid[kc];
        }
      }
      k0 += __popc(sm);
    }
    if (lane == 0) B.val[6] = k0;
  }
  for (int f = tid; f < nf; f += nt) {
    const unsigned fw = P.fnew[f];
    if (fw != C::FNONE) {
      P.fs[nb][fw] = P.fns[f];
      P.fn[nb][fw] = P.fn[cb][f];
    }
  }
  if (tid == 0) P.fs[nb][nfk] = (typename C::Pos)hk;
  __syncthreads();
  const int nseg = B.val[6];
  if (nseg > C::SCAP) return kClipOverflow;

  // 8. the lid (:470-495), warp 0: lid_map (last writer wins) and the chain
  //    from the first segment, appended as the last face
  if (w == 0) {
    int len = 0, ovf = 0;
    if (nseg > 0) {
      for (int v = nkept + lane; v < nvn; v += 32) P.lidmap[v] = (VId)C::VNONE;
      __syncwarp();
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
      if (!ovf && len >= 3) {
        if (nfk + 1 > C::FCAP || len > 255) {
          ovf = 1;
        } else {
          for (int q = lane; q < len; q += 32) P.pf[nb][hk + q] = (FId)nfk;
          if (lane == 0) {
            P.fs[nb][nfk] = (typename C::Pos)hk;
            P.fn[nb][nfk] = nbr;
            P.fs[nb][nfk + 1] = (typename C::Pos)(hk + len);
          }
        }
      }
    }
    if (lane == 0) {
      B.val[7] = ovf ? -1 : len;
    }
  }
  // the clip's max radius: every thread's kept and new vertices
  const double wr = warp_max(r2);
  if (lane == 0) B.r2[w] = wr;
  __syncthreads();
  const int lidlen = B.val[7];
  double rm = 0.0;
  for (int q = 0; q < NW; ++q) rm = fmax(rm, B.r2[q]);
  __syncthreads();  // B is reused by the next clip
  if (lidlen < 0) return kClipOverflow;
  S.nv = nvn;
  S.nf = lidlen >= 3 ? nfk + 1 : nfk;
  S.nh = lidlen >= 3 ? hk + lidlen : hk;
  S.cb = nb;
  *r2out = with_gen ? rm : 0.0;
  return kClipMod;
}

// compute_cell (tessellation.rs:414-475) over a block-wide polytope X: the
// walls' planes, then the candidates in search order.  The walk runs in every
// warp (same data, same decisions, a staging row per warp) and all warps enter
// each clip together.  X provides init (the box), clip (clip_with_scratch's
// result and the new largest radius), empty and max_radius; the layouts that
// use it give the same results, bit for bit.
template <int NW, class X>
__device__ int block_walk(const TessDesc& T, uint32_t i, BlockShared<NW>& B, X& poly) {
  const unsigned lane = lane_id();
  const double gx = T.gen[3 * (size_t)i], gy = T.gen[3 * (size_t)i + 1], gz = T.gen[3 * (size_t)i + 2];
  double r2;
  poly.init(T.grid, gx, gy, gz);
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
        const int r = poly.clip(p[0], p[1], p[2], n[0], n[1], n[2], W.id, false, gx, gy, gz, &r2);
        if (r == kClipOverflow) return kCellOverflow;
      }
    }
    if (poly.empty()) return kCellOk;
  }
  double cur = poly.max_radius(gx, gy, gz);

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
  for (int base = 0; base < T.norder && !done; base += 32) {
    // ---- this lane's search-order entry ----
    const int k = base + (int)lane;
    const bool valid = k < T.norder;
    double md2 = 0.0, b2 = 0.0;
    bool inr = false;
    uint32_t bs = 0, be = 0;
    if (valid) {
      const Offset o = T.order[k];
      md2 = o.min_d2;
      const int bx = ix + o.dx, by = iy + o.dy, bz = iz + o.dz;
      inr = bx >= 0 && bx < G.n[0] && by >= 0 && by < G.n[1] && bz >= 0 && bz < G.n[2];
      if (inr) {
        const double ddx = o.dx > 0 ? ((double)o.dx - rx) * G.cs[0]
                                    : (o.dx < 0 ? ((double)(-(o.dx + 1)) + rx) * G.cs[0] : 0.0);
        const double ddy = o.dy > 0 ? ((double)o.dy - ry) * G.cs[1]
                                    : (o.dy < 0 ? ((double)(-(o.dy + 1)) + ry) * G.cs[1] : 0.0);
        const double ddz = o.dz > 0 ? ((double)o.dz - rz) * G.cs[2]
                                    : (o.dz < 0 ? ((double)(-(o.dz + 1)) + rz) * G.cs[2] : 0.0);
        const double bdx = fmax(ddx, 0.0), bdy = fmax(ddy, 0.0), bdz = fmax(ddz, 0.0);
        b2 = bdx * bdx + bdy * bdy + bdz * bdz;
        const uint32_t bb = (uint32_t)bx + (uint32_t)by * (uint32_t)G.n[0] + (uint32_t)bz * nxy;
        // on sparse grids an empty bin is known from its occupancy bit (an
        // L2-resident map) without reading the bin table
        if (!T.occ || ((__ldg(&T.occ[bb >> 5]) >> (bb & 31u)) & 1u)) {
          bs = T.bin_start[bb];
          be = T.bin_start[bb + 1];
        }
      }
    }
    // bins that can still open (R only shrinks), flattened: members of entry
    // e are candidates [start, start + cnt)
    const bool pot = valid && inr && be > bs && !(md2 > 4.0 * cur) && b2 <= 4.0 * cur;
    if (!__any_sync(kFull, pot)) {
      // no bin of this chunk can open (sparse regions, fine grids): only
      // the end of the walk is decided here
      const unsigned brk = __ballot_sync(kFull, valid && md2 > 4.0 * cur);
      const int fbe = brk ? __ffs(brk) - 1 : 32;
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
        for (int q = lo; q < hi; ++q) B.cand[threadIdx.x >> 5][q - r0] = (uint8_t)lane;
      }
      __syncwarp();
      const int idx = r0 + (int)lane;
      const bool have = idx < total;
      const int ce = have ? (int)B.cand[threadIdx.x >> 5][lane] : 0;
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
        const int j = __ffs(pass) - 1;
        const int ej = __shfl_sync(kFull, ce, j);
        const int jid = (int)__shfl_sync(kFull, sg.id, j);
        const double e0 = __shfl_sync(kFull, d0, j);
        const double e1 = __shfl_sync(kFull, d1, j);
        const double e2 = __shfl_sync(kFull, d2, j);
        const double mx = gx + e0 * 0.5, my = gy + e1 * 0.5, mz = gz + e2 * 0.5;
        const int r = poly.clip(mx, my, mz, e0, e1, e2, jid, true, gx, gy, gz, &r2);
        if (r == kClipOverflow) return kCellOverflow;
        if (r == kClipMod) cur = r2;
        else if (r == kClipEmpty) cur = 0.0;
        ecur = ej;
        pos = r0 + j + 1;
      }
      if (r0 + 32 >= total) break;
      // the next round starts at an entry the walk no longer reaches
      const unsigned nxt = __ballot_sync(kFull, cnt > 0 && start <= r0 + 32);
      if (fb < 32 && 31 - __clz(nxt) >= fb) break;
    }
    if (fb < 32) done = true;
  }
  if (!done && !T.order_complete && !(T.order_bound > 4.0 * cur)) return kCellTable;
  return kCellOk;
}


// the full-rewrite layout's operations for block_walk
template <class C, int NW>
struct BlockPolyOps {
  WarpPoly<C>& P;
  BlockShared<NW>& B;
  PolyState& S;
  __device__ void init(const Grid& g, double gx, double gy, double gz) {
    // the box, written by warp 0; every thread holds the same state
    if ((threadIdx.x >> 5) == 0) poly_init_box(P, S, g, gx, gy, gz);
    S.nv = 8;
    S.nf = 6;
    S.nh = 24;
    S.cb = 0;
    S.umax = 0.0;
    __syncthreads();
  }
  __device__ int clip(double px, double py, double pz, double nx, double ny, double nz, int nbr, bool with_gen,
                      double gx, double gy, double gz, double* r2out) {
    return block_clip<C, NW>(P, B, S, px, py, pz, nx, ny, nz, nbr, with_gen, gx, gy, gz, r2out);
  }
  __device__ bool empty() const { return S.nv == 0; }
  __device__ double max_radius(double gx, double gy, double gz) { return poly_max_radius_sq(P, S, gx, gy, gz); }
};

// compute_cell by a whole block on the full-rewrite layout
template <class C, int NW>
__device__ int compute_cell_block(const TessDesc& T, uint32_t i, WarpPoly<C>& P, BlockShared<NW>& B,
                                   PolyState& S) {
  BlockPolyOps<C, NW> ops{P, B, S};
  return block_walk<NW>(T, i, B, ops);
}

constexpr int kHugeBlockWarps = 32;
// the narrower blocks (the host's default width for the huge tier, a tuning
// setting; the width changes no result): on the slot layout the clip's
// one-warp rewrite and its barriers, not the classification's passes, set the
// time, and 16 warps win at every size measured (the centre of 3,000 /
// 10,000 / 20,000 generators on a sphere: 30.4 / 147.6 / 435 ms against 38.1 /
// 163.8 / 450 ms with 32, and 35.1 / 204 / 655 ms with 8, too few warps for
// the classification's pass)
constexpr int kHugeBlockWarpsNarrow = 16;

}  // namespace vd
