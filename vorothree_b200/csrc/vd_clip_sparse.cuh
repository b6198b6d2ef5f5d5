// vd_clip_sparse.cuh -- the shared-memory tier's polytope with stable vertex
// slots: a modifying clip rewrites only the faces that lose a vertex.
//
// Cell3DFaces::clip_with_scratch (cell_3d_faces.rs:288-503) rebuilds the whole
// vertex list and every face loop on each modifying clip.  What it produces
// depends on the clip history only through these facts, which this layout
// keeps instead of the rebuilt arrays:
//  * vertex identity -- the intersection map and the lid map look vertices up
//    by id, and the kept vertices keep their coordinates.  Here each vertex
//    lives in a fixed slot until it is cut away; a cut-away vertex's slot is
//    reused by a new intersection vertex.  (The reference's vertex ORDER --
//    kept vertices first, then intersections in discovery order -- matters
//    only to a polytope export, which the other tiers do.)
//  * face order -- surviving faces in their order, the lid last: kept here as
//    a compacted face table.
//  * each face's loop, including where it starts: a face with no vertex
//    outside the plane comes back from the reference's face walk rotated by
//    one entry (each in->in edge emits its end vertex).  Here such a face is
//    not touched; its rotation counter goes up by one.  Only a face with an
//    outside vertex is walked, from its logical first entry, exactly as the
//    reference walks it, into fresh entries.
// Each face carries a 96-bit mask of its vertex slots, so the faces a clip
// touches are found with three AND operations per face.
//
// Only the general case is handled: every touched face has exactly two
// crossing edges (one in->out, one out->in), every crossing edge is shared by
// two touched faces, and the lid segments form one cycle (or cycles the
// reference's chain walk follows from its first segment).  Anything else --
// degenerate configurations where vertices sit within the 1e-9 band -- and
// any capacity overflow returns kClipOverflow, and the cell is rebuilt from
// scratch by the medium tier's full clip (vd_clip.cuh), whose results are
// the reference's in every case.  Both produce the same doubles in the same
// order, so results do not depend on which tier finished a cell.
#pragma once
#include "vd_clip.cuh"

namespace vd {

template <int V, int F, int E, bool kCount, bool kMixed>
struct SparseCfg {
  static constexpr bool COUNT = kCount;
  static constexpr bool MIXED = kMixed;
  static constexpr int VCAP = V;   // vertex slots (three 32-bit mask words)
  static constexpr int FCAP = F;   // faces (one lane each)
  static constexpr int ECAP = E;   // face entries per entry buffer
  static constexpr int XCAP = 32;  // crossing edges per clip (one lane each)
  static constexpr int TCAP = 256; // edges of the touched faces per clip (32 per round)
  static_assert(V > 64 && V <= 96, "vertex slots take three 32-bit mask words");
  static_assert(V < 255, "vertex slots are bytes; 255 marks an empty lid-map entry");
  static_assert(F <= 32, "one lane per face");
  static_assert(E <= 65535, "16-bit entry offsets");
};

// capacities: 96 vertex slots, 32 faces, 256 entries -- the fast tier's
// shared-memory budget; larger polytopes (rare for uniform input: at most 72
// vertices and 38 faces over 7.5 M cells) overflow to the medium tier
using FastSparse = SparseCfg<96, 32, 256, false, false>;
using FastSparseCount = SparseCfg<96, 32, 256, true, false>;
using MixedSparse = SparseCfg<96, 32, 256, false, true>;
using MixedSparseCount = SparseCfg<96, 32, 256, true, true>;

struct SparseState {
  int nf;      // faces
  int hw;      // slots [0, hw) may be live
  int cb;      // entry buffer holding the faces' entries
  int etop;    // first unused entry of that buffer
  unsigned live0, live1, live2;  // live vertex slots
  double umax;  // mixed path: bound on |v - g|_inf over the live vertices
};

__device__ __forceinline__ bool state_empty(const SparseState& S) { return (S.live0 | S.live1 | S.live2) == 0u; }

template <class C>
struct alignas(16) SparsePoly {
  using State = SparseState;
  static constexpr bool kExport = false;  // vertex slots are not in the reference's order
  double vx[C::VCAP], vy[C::VCAP], vz[C::VCAP];
  double vr2[C::VCAP];  // |v - g|^2 (the radius the clip returns), set when the vertex is made
  double dist[C::MIXED ? 1 : C::VCAP];  // plain path: signed distances of the current clip
  // mixed path: FP32 generator-relative copies and their max norm
  float ux[C::MIXED ? C::VCAP : 1], uy[C::MIXED ? C::VCAP : 1], uz[C::MIXED ? C::VCAP : 1];
  float uin[C::MIXED ? C::VCAP : 1];
  unsigned long long cnt[C::COUNT ? kNumCounters : 1];
  int32_t fn[C::FCAP];                               // face neighbour id
  unsigned fm0[C::FCAP], fm1[C::FCAP], fm2[C::FCAP];  // vertex slots of each face
  uint16_t fst[C::FCAP];                             // first entry of the face in the entry buffer
  uint8_t fc[C::FCAP];                               // entry count
  uint8_t fr[C::FCAP];                               // rotation: logical entry j is ent[fst + (j + fr) % fc]
  uint8_t ent[2][C::ECAP];                           // face entries (vertex slots); the second buffer for compaction
  // per clip: the crossing edges in walk order (touched faces in face order,
  // each from its logical first entry); touched face k's two are 2k, 2k+1
  uint16_t xkey[C::XCAP];  // (min, max) slot pair of the edge
  uint8_t xs[C::XCAP], xe[C::XCAP];  // the edge as the face walks it
  uint16_t xpos[C::XCAP];  // entry that receives the intersection vertex; finalize: first triangle of face g
  uint8_t xt[C::XCAP];     // 1: in->out, 0: out->in
  uint8_t xf[C::XCAP];     // rank of the crossing's face among the touched faces
  uint8_t tmap[32];        // face of each touched-face rank
  uint8_t freel[C::VCAP];   // per clip: the free slots in order
  uint8_t cand_e[32];  // walk: search-order entry of each candidate of a round
};

template <class C>
__device__ __forceinline__ void cnt_add(SparsePoly<C>& P, int k, unsigned long long v) {
  if constexpr (C::COUNT) {
    if (lane_id() == 0) P.cnt[k] += v;
  }
}

__device__ __forceinline__ unsigned sp_word(unsigned a, unsigned b, unsigned c, unsigned s) {
  return s < 32u ? a : (s < 64u ? b : c);
}

__device__ __forceinline__ bool sp_bit(unsigned a, unsigned b, unsigned c, unsigned s) {
  return (sp_word(a, b, c, s) >> (s & 31u)) & 1u;
}

// Cell3DFaces::new (cell_3d_faces.rs:37-74): the box, faces z-, z+, y-, y+,
// x-, x+ with ids box_side (bounds/mod.rs:21-22)
template <class C>
__device__ void poly_init_box(SparsePoly<C>& P, SparseState& S, const Grid& g, double gx, double gy, double gz) {
  const unsigned lane = lane_id();
  float um = 0.f;
  if (lane < 8) {
    const unsigned hx = (lane == 1 || lane == 2 || lane == 5 || lane == 6);
    const unsigned hy = (lane == 2 || lane == 3 || lane == 6 || lane == 7);
    const unsigned hz = lane >= 4;
    const double x = hx ? g.bmax[0] : g.bmin[0];
    const double y = hy ? g.bmax[1] : g.bmin[1];
    const double z = hz ? g.bmax[2] : g.bmin[2];
    P.vx[lane] = x;
    P.vy[lane] = y;
    P.vz[lane] = z;
    const double dx = x - gx, dy = y - gy, dz = z - gz;
    P.vr2[lane] = dx * dx + dy * dy + dz * dz;
    if constexpr (C::MIXED) {
      const float fx = (float)dx, fy = (float)dy, fz = (float)dz;
      P.ux[lane] = fx;
      P.uy[lane] = fy;
      P.uz[lane] = fz;
      um = fmaxf(fabsf(fx), fmaxf(fabsf(fy), fabsf(fz)));
      P.uin[lane] = um;
    }
  }
  // face loops 3210 4567 0154 2376 0473 1265 packed as nibbles, lane = entry
  constexpr unsigned long long lo = 0x6732451076540123ull, hi = 0x56213740ull;
  if (lane < 24) {
    const unsigned idx = (unsigned)((lane < 16 ? lo >> (4 * lane) : hi >> (4 * (lane - 16))) & 0xFull);
    P.ent[0][lane] = (uint8_t)idx;
  }
  if (lane < 6) {
    unsigned m = 0;
    for (unsigned q = 4 * lane; q < 4 * lane + 4; ++q)
      m |= 1u << (unsigned)((q < 16 ? lo >> (4 * q) : hi >> (4 * (q - 16))) & 0xFull);
    P.fm0[lane] = m;
    P.fm1[lane] = 0u;
    P.fm2[lane] = 0u;
    P.fst[lane] = (uint16_t)(4 * lane);
    P.fc[lane] = 4;
    P.fr[lane] = 0;
    // face ids z-, z+, y-, y+, x-, x+ = box_side(axis, is_max) = -1 - (2*axis + is_max)
    P.fn[lane] = -1 - (2 * (2 - (int)(lane >> 1)) + (int)(lane & 1));
  }
  S.nf = 6;
  S.hw = 8;
  S.cb = 0;
  S.etop = 24;
  S.live0 = 0xFFu;
  S.live1 = 0u;
  S.live2 = 0u;
  S.umax = 0.0;
  if constexpr (C::MIXED) {
    double m = (double)um;
    S.umax = warp_max(m) * (1.0 + 0x1p-20);
  }
  __syncwarp();
}

// max_radius_sq (cell_3d_faces.rs:271-286): the largest |v - g|^2 over the
// live vertices (each computed with the reference's expression when the
// vertex was made; a maximum does not depend on the order it is taken in)
template <class C>
__device__ double poly_max_radius_sq(const SparsePoly<C>& P, const SparseState& S, double, double, double) {
  const unsigned lane = lane_id();
  double m = 0.0;
#pragma unroll
  for (int w = 0; w < 3; ++w) {
    const unsigned Lw = w == 0 ? S.live0 : (w == 1 ? S.live1 : S.live2);
    if ((Lw >> lane) & 1u) m = fmax(m, P.vr2[32 * w + lane]);
  }
  return sp_warp_max_nonneg(m);
}

// whether clip_with_scratch with this lane's own plane would change the
// polytope: some live vertex outside, d > 1e-9, computed as the clip does
// (every lane walks every live slot in the same order)
template <class C>
__device__ __forceinline__ bool plane_cuts(const SparsePoly<C>& P, const SparseState& S, double px, double py,
                                           double pz, double nx, double ny, double nz) {
  bool cut = false;
#pragma unroll
  for (int w = 0; w < 3; ++w) {
    unsigned L = w == 0 ? S.live0 : (w == 1 ? S.live1 : S.live2);
    while (L) {
      const int v = 32 * w + __ffs(L) - 1;
      L &= L - 1u;
      const double d = (P.vx[v] - px) * nx + (P.vy[v] - py) * ny + (P.vz[v] - pz) * nz;
      cut |= d > kTol;
    }
  }
  return cut;
}

template <class C>
__device__ __forceinline__ int poly_nverts(const SparsePoly<C>&, const SparseState& S) {
  return __popc(S.live0) + __popc(S.live1) + __popc(S.live2);
}

// clip_with_scratch (cell_3d_faces.rs:288-503) on the slot layout.  All lanes
// call it with the same arguments; the return value and *r2out are the
// reference's (*r2out: the largest |v - g|^2 over the new vertex set when
// with_gen, else 0).
template <class C>
__device__ int warp_clip(SparsePoly<C>& P, SparseState& S, double px, double py, double pz, double nx, double ny,
                         double nz, int nbr, bool with_gen, double gx, double gy, double gz, double* r2out) {
  const unsigned lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  const unsigned L0 = S.live0, L1 = S.live1, L2 = S.live2;
  const int hw = S.hw;
  cnt_add(P, kCntClips, 1);
  cnt_add(P, kCntClassified, (unsigned long long)(__popc(L0) + __popc(L1) + __popc(L2)));

  // 1. signed distances of the live vertices and the 3-band flags (:302-326)
  unsigned O0 = 0u, O1 = 0u, O2 = 0u;
  bool sin = false;
  {
    float hi_out = 0.f, lo_sin = 0.f, band_lo = 0.f, band_hi = 0.f;
    float fnx = 0.f, fny = 0.f, fnz = 0.f, fc = 0.f;
    bool fp32_ok = false;
    if constexpr (C::MIXED) {
      // FP32 distance on generator-relative coordinates, d32 = u.n - c with
      // c = (p - g).n.  Forward error bound against the FP64 value
      // d64 = (v - p).n (u = fl32(fl64(v - g))):
      //   |d32 - d64| <= 2^-21 (|u|_inf |n|_1 + |c| + sum_k |(p_k - g_k) n_k|) + 1e-30.
      // A vertex whose d32 lies within that bound of +-1e-9 is re-evaluated
      // with the FP64 formula, so every decision equals the plain path's.
      const double qx = px - gx, qy = py - gy, qz = pz - gz;
      const double c = qx * nx + qy * ny + qz * nz;
      const double qn = fabs(qx * nx) + fabs(qy * ny) + fabs(qz * nz);
      const double scale = S.umax * (fabs(nx) + fabs(ny) + fabs(nz)) + fabs(c);
      const double bound = 0x1p-21 * (scale + qn) + 1e-30;
      fp32_ok = scale > 1e-24 && scale < 1e24;
      fnx = (float)nx;
      fny = (float)ny;
      fnz = (float)nz;
      fc = (float)c;
      // the thresholds rounded outward (out/inside) and the exact-free band
      // rounded inward, so comparing the FP32 value with them decides no
      // vertex that the FP64 comparison would decide differently
      hi_out = __double2float_ru(kTol + bound);
      lo_sin = __double2float_rd(-kTol - bound);
      band_lo = __double2float_ru(-kTol + bound);
      band_hi = __double2float_rd(kTol - bound);
    }
#pragma unroll
    for (int w = 0; w < 3; ++w) {
      if (32 * w < hw) {
        const unsigned Lw = w == 0 ? L0 : (w == 1 ? L1 : L2);
        const int v = 32 * w + (int)lane;
        bool o = false, si = false;
        if ((Lw >> lane) & 1u) {
          if constexpr (!C::MIXED) {
            const double d = (P.vx[v] - px) * nx + (P.vy[v] - py) * ny + (P.vz[v] - pz) * nz;
            P.dist[v] = d;
            o = d > kTol;
            si = d < -kTol;
          } else {
            bool exact = !fp32_ok;
            if (fp32_ok) {
              const float d32 = fmaf(P.ux[v], fnx, fmaf(P.uy[v], fny, P.uz[v] * fnz)) - fc;
              if (d32 > hi_out) o = true;
              else if (d32 < lo_sin) si = true;
              else exact = !(d32 >= band_lo && d32 <= band_hi);
            }
            if (exact) {
              const double d = (P.vx[v] - px) * nx + (P.vy[v] - py) * ny + (P.vz[v] - pz) * nz;
              o = d > kTol;
              si = d < -kTol;
            }
          }
        }
        const unsigned om = __ballot_sync(kFull, o);
        if (w == 0) O0 = om;
        else if (w == 1) O1 = om;
        else O2 = om;
        sin |= si;
      }
    }
  }
  if (!(O0 | O1 | O2)) {
    *r2out = 0.0;
    return kClipNoop;
  }
  if (!__any_sync(kFull, sin)) {
    S.live0 = S.live1 = S.live2 = 0u;
    S.nf = 0;
    S.hw = 0;
    S.etop = 0;
    *r2out = 0.0;
    return kClipEmpty;
  }
  cnt_add(P, kCntModifying, 1);
  // kept vertices (d <= 1e-9, :344-362)
  const unsigned I0 = L0 & ~O0, I1 = L1 & ~O1, I2 = L2 & ~O2;

  // 2. faces, one lane each: a face with a kept vertex survives; one that
  //    also has an outside vertex is touched (walked and rewritten)
  const int nf = S.nf;
  const int src = S.cb;
  const bool fv = (int)lane < nf;
  unsigned m0 = 0u, m1 = 0u, m2 = 0u;
  int c = 0, st = 0, rot = 0;
  if (fv) {
    m0 = P.fm0[lane];
    m1 = P.fm1[lane];
    m2 = P.fm2[lane];
    c = P.fc[lane];
    st = P.fst[lane];
    rot = P.fr[lane];
  }
  const bool kept = fv && ((m0 & I0) | (m1 & I1) | (m2 & I2)) != 0u;
  const bool touched = kept && ((m0 & O0) | (m1 & O1) | (m2 & O2)) != 0u;
  const unsigned km = __ballot_sync(kFull, kept);
  const unsigned tm = __ballot_sync(kFull, touched);
  const int nkeep = __popc(km), ntouch = __popc(tm);
  if (ntouch < 3 || 2 * ntouch > C::XCAP || nkeep + 1 > C::FCAP) return kClipOverflow;
  const int trank = __popc(tm & lt), fnew = __popc(km & lt);
  // a touched face keeps all its kept vertices and gains two intersections
  const int nsz = touched ? __popc(m0 & I0) + __popc(m1 & I1) + __popc(m2 & I2) + 2 : 0;
  const int incl = warp_incl_scan(nsz);
  const int eoff = incl - nsz;
  const int tot_new = __shfl_sync(kFull, incl, 31);
  const int need = tot_new + ntouch;  // the touched faces and the lid (at most one entry per segment)

  // entry space: append after the live entries, or copy the untouched faces
  // (in logical order) to the front of the other buffer first
  int dst = src, base = S.etop;
  if (base + need > C::ECAP) {
    const int csz = (kept && !touched) ? c : 0;
    const int cinc = warp_incl_scan(csz);
    base = __shfl_sync(kFull, cinc, 31);
    if (base + need > C::ECAP) return kClipOverflow;
    dst = src ^ 1;
    if (csz) {
      const int cofs = cinc - csz;
      int q = rot;
      for (int j = 0; j < c; ++j) {
        P.ent[dst][cofs + j] = P.ent[src][st + q];
        q = (q + 1 == c) ? 0 : q + 1;
      }
      // the face's table entry now points at its logical-order copy (only
      // this lane reads it again)
      P.fst[lane] = (uint16_t)cofs;
      P.fr[lane] = 0;
    }
  }

  // 3. the touched faces' edges in walk order (faces in order, each from its
  //    logical first entry), one lane per edge, 32 per round -- the face walk
  //    of :369-452: in->in emits the end, in->out the intersection, out->in
  //    the intersection and the end.  The new faces follow one another in
  //    face order, so an emitted entry's place is the running count of the
  //    entries emitted before it.  Crossings are listed in walk order.
  {
    const int tsz = touched ? c : 0;
    const int tinc = warp_incl_scan(tsz);
    const int tpos0 = tinc - tsz;
    const int np = __shfl_sync(kFull, tinc, 31);
    if (np > C::TCAP) return kClipOverflow;
    if (touched) P.tmap[trank] = (uint8_t)lane;
    __syncwarp();
    uint8_t* D = P.ent[dst];
    const int dend = base + tot_new;
    int run = base, ncr = 0;
    for (int r0 = 0; r0 < np; r0 += 32) {
      const int i = r0 + (int)lane;
      const bool act = i < np;
      // the face of edge i: the touched faces that start at or before it (a
      // start bit per face starting in this round, a count for the earlier
      // ones)
      const unsigned sb = __reduce_or_sync(
          kFull, (touched && tpos0 >= r0 && tpos0 < r0 + 32) ? 1u << (tpos0 - r0) : 0u);
      const int before = __popc(__ballot_sync(kFull, touched && tpos0 < r0));
      const int rk = before + __popc(sb & (lane == 31 ? kFull : (2u << lane) - 1u)) - 1;
      const int f = act ? P.tmap[rk] : 0;
      const int fst0 = __shfl_sync(kFull, st, f), frot = __shfl_sync(kFull, rot, f);
      const int fcn = __shfl_sync(kFull, c, f), ftp = __shfl_sync(kFull, tpos0, f);
      const int frank = __shfl_sync(kFull, trank, f);
      unsigned sv = 0, ev = 0;
      bool si = false, ei = false;
      if (act) {
        int q = i - ftp + frot;
        if (q >= fcn) q -= fcn;
        const int q2 = (q + 1 == fcn) ? 0 : q + 1;
        sv = P.ent[src][fst0 + q];
        ev = P.ent[src][fst0 + q2];
        si = sp_bit(I0, I1, I2, sv);
        ei = sp_bit(I0, I1, I2, ev);
      }
      const int emit = act ? (si ? 1 : (ei ? 2 : 0)) : 0;
      const int einc = warp_incl_scan(emit);
      const int idx = run + einc - emit;
      const bool cr = act && si != ei;
      const unsigned cm = __ballot_sync(kFull, cr);
      if (cr) {
        const int g = ncr + __popc(cm & lt);
        if (g < C::XCAP) {
          P.xkey[g] = (uint16_t)(sv < ev ? (sv << 8 | ev) : (ev << 8 | sv));
          P.xs[g] = (uint8_t)sv;
          P.xe[g] = (uint8_t)ev;
          P.xpos[g] = (uint16_t)idx;  // the intersection's entry, written once its slot is known
          P.xt[g] = si ? 1 : 0;
          P.xf[g] = (uint8_t)frank;
        }
      }
      if (ei) {
        const int k = idx + (si ? 0 : 1);
        if (k < dend) D[k] = (uint8_t)ev;
      }
      run += __shfl_sync(kFull, einc, 31);
      ncr += __popc(cm);
    }
    // every touched face has one in->out and one out->in crossing (then it
    // emitted exactly its kept vertices and two intersections)
    if (run != dend || ncr != 2 * ntouch) return kClipOverflow;
  }
  __syncwarp();

  // 4. intersection vertices: crossing g is lane g; the first of the two
  //    crossings of an edge in walk order (face order, then walk position)
  //    creates the vertex from its own walk direction, the other reuses it
  //    (the intersection_map of :391-417 / :422-448)
  const int ncross = 2 * ntouch;
  const bool act = (int)lane < ncross;
  // crossings 2k and 2k+1 belong to touched face k, one of each direction
  const unsigned tg = act ? (unsigned)P.xt[lane] : 0u;
  const unsigned tother = __shfl_xor_sync(kFull, tg, 1);
  if (__any_sync(kFull, act && ((int)P.xf[lane] != ((int)lane >> 1) || tg == tother))) return kClipOverflow;
  const unsigned key = act ? (unsigned)P.xkey[lane] : (0xFFFF0000u | lane);
  const unsigned mm = __match_any_sync(kFull, key);
  const int leader = __ffs(mm) - 1;
  const bool isl = act && leader == (int)lane;
  if (__any_sync(kFull, act && __popc(mm) != 2)) return kClipOverflow;
  // the other crossing of the same edge: the neighbouring touched face walks
  // the edge the other way, so an in->out crossing's partner is out->in
  const int partner = act ? __ffs(mm & ~(1u << lane)) - 1 : (int)lane;
  const unsigned ptg = __shfl_sync(kFull, tg, partner & 31);  // every lane shuffles
  if (__any_sync(kFull, act && tg == ptg)) return kClipOverflow;
  const unsigned dm = __ballot_sync(kFull, isl);
  cnt_add(P, kCntIntersections, (unsigned long long)__popc(dm));
  // the new vertex of discovery rank r takes the r-th free slot (cut-away
  //    slots are free again): the free slots listed in order, word by word,
  //    as far as the new vertices need
  const int nnew = __popc(dm);
  {
    unsigned F2 = ~I2;
    if constexpr (C::VCAP < 96) F2 &= (1u << (C::VCAP < 96 ? C::VCAP - 64 : 0)) - 1u;
    const unsigned F0 = ~I0, F1 = ~I1;
    const int c0 = __popc(F0), c1 = __popc(F1), c2 = __popc(F2);
    if (nnew > c0 + c1 + c2) return kClipOverflow;
    if ((F0 >> lane) & 1u) P.freel[__popc(F0 & lt)] = (uint8_t)lane;
    if (nnew > c0) {
      if ((F1 >> lane) & 1u) P.freel[c0 + __popc(F1 & lt)] = (uint8_t)(32 + lane);
      if (nnew > c0 + c1 && ((F2 >> lane) & 1u)) P.freel[c0 + c1 + __popc(F2 & lt)] = (uint8_t)(64 + lane);
    }
    __syncwarp();
  }
  const int slot = isl ? (int)P.freel[__popc(dm & lt)] : -1;
  double ix = 0.0, iy = 0.0, iz = 0.0, d2 = 0.0;
  if (isl) {
    const unsigned s = P.xs[lane], e = P.xe[lane];
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
    ix = ax + t * (bx - ax);
    iy = ay + t * (by - ay);
    iz = az + t * (bz - az);
    const double dx = ix - gx, dy = iy - gy, dz = iz - gz;
    d2 = dx * dx + dy * dy + dz * dz;
  }
  __syncwarp();  // every endpoint is read before a slot it frees is reused
  if (isl) {
    P.vx[slot] = ix;
    P.vy[slot] = iy;
    P.vz[slot] = iz;
    P.vr2[slot] = d2;
    if constexpr (C::MIXED) {
      const float fx = (float)(ix - gx), fy = (float)(iy - gy), fz = (float)(iz - gz);
      P.ux[slot] = fx;
      P.uy[slot] = fy;
      P.uz[slot] = fz;
      P.uin[slot] = fmaxf(fabsf(fx), fmaxf(fabsf(fy), fabsf(fz)));
    }
  }
  const int id = __shfl_sync(kFull, slot, leader);
  if (act) P.ent[dst][P.xpos[lane]] = (uint8_t)id;
  // the new vertices took the free slots up to the last one's: the lowest
  // nnew free slots
  unsigned N0, N1, N2;
  int nhw;
  {
    const int sl = P.freel[nnew - 1];  // (nnew >= 3: a touched face has two crossings, three faces at least)
    unsigned F2 = ~I2;
    if constexpr (C::VCAP < 96) F2 &= (1u << (C::VCAP < 96 ? C::VCAP - 64 : 0)) - 1u;
    auto upto = [](int b) { return b >= 31 ? kFull : (2u << b) - 1u; };  // bits 0..b of a word
    N0 = ~I0 & (sl >= 32 ? kFull : upto(sl));
    N1 = sl < 32 ? 0u : (~I1 & (sl >= 64 ? kFull : upto(sl - 32)));
    N2 = sl < 64 ? 0u : (F2 & upto(sl - 64));
    nhw = max(hw, sl + 1);
  }

  // 5. the lid (:470-495): touched face k gives the segment (X of its
  //    out->in crossing, X of its in->out crossing), and lid_map[start] = end.
  //    The end of segment k is the intersection on its in->out edge, which
  //    is the out->in intersection -- the start -- of the face across that
  //    edge: the segment that follows k in the chain is the face of its
  //    in->out crossing's partner.  Every face has one crossing of each
  //    direction and crossings pair up, so the successors form a
  //    permutation; the chain from segment 0 is ranked by pointer jumping.
  const bool sact = (int)lane < ntouch;
  const int id0 = __shfl_sync(kFull, id, (2 * (int)lane) & 31);
  const int id1 = __shfl_sync(kFull, id, (2 * (int)lane + 1) & 31);
  const bool io0 = __shfl_sync(kFull, tg, (2 * (int)lane) & 31) != 0u;  // crossing 2k is the in->out one
  const unsigned a = (unsigned)(io0 ? id1 : id0);
  const int pio = __shfl_sync(kFull, partner, (2 * (int)lane + (io0 ? 0 : 1)) & 31);
  const unsigned succ = sact ? (unsigned)(pio >> 1) : lane;
  const int term = __ffs(__ballot_sync(kFull, sact && succ == 0u)) - 1;
  int nxt = (sact && (int)lane != term) ? (int)succ : (int)lane;
  int dd = nxt != (int)lane ? 1 : 0;
  for (int span = 1; span < ntouch; span <<= 1) {
    const int dn = __shfl_sync(kFull, dd, nxt);
    const int nn = __shfl_sync(kFull, nxt, nxt);
    dd += dn;
    nxt = nn;
  }
  const int d0 = __shfl_sync(kFull, dd, 0);
  const int len = d0 + 1;
  const bool oncyc = sact && nxt == term;
  const int lbase = base + tot_new;
  if (oncyc) P.ent[dst][lbase + d0 - dd] = (uint8_t)a;
  const bool addlid = len >= 3;
  const unsigned A0 = __reduce_or_sync(kFull, (oncyc && a < 32u) ? 1u << a : 0u);
  const unsigned A1 = __reduce_or_sync(kFull, (oncyc && a >= 32u && a < 64u) ? 1u << (a - 32u) : 0u);
  const unsigned A2 = __reduce_or_sync(kFull, (oncyc && a >= 64u && a < 96u) ? 1u << (a - 64u) : 0u);

  // 6. the face table: surviving faces in order, then the lid
  //    (each lane reads its face's entry again rather than keeping it in
  //    registers through steps 3-5)
  const int xk0 = __shfl_sync(kFull, id, (2 * trank) & 31);
  const int xk1 = __shfl_sync(kFull, id, (2 * trank + 1) & 31);
  const bool kio0 = __shfl_sync(kFull, tg, (2 * trank) & 31) != 0u;
  const int xio = kio0 ? xk0 : xk1;
  const int xoi = kio0 ? xk1 : xk0;
  int nst = 0, nc = 0, nr = 0, fnv = 0;
  unsigned w0 = 0u, w1 = 0u, w2 = 0u;
  if (kept) {
    fnv = P.fn[lane];
    w0 = P.fm0[lane];
    w1 = P.fm1[lane];
    w2 = P.fm2[lane];
    nst = P.fst[lane];
    nc = P.fc[lane];
    const int fr0 = P.fr[lane];
    nr = (fr0 + 1 == nc) ? 0 : fr0 + 1;
  }
  if (touched) {
    nst = base + eoff;
    nc = nsz;
    nr = 0;
    w0 &= I0;
    w1 &= I1;
    w2 &= I2;
    if (xio < 32) w0 |= 1u << xio;
    else if (xio < 64) w1 |= 1u << (xio - 32);
    else w2 |= 1u << (xio - 64);
    if (xoi < 32) w0 |= 1u << xoi;
    else if (xoi < 64) w1 |= 1u << (xoi - 32);
    else w2 |= 1u << (xoi - 64);
  }
  __syncwarp();
  if (kept) {
    P.fn[fnew] = fnv;
    P.fst[fnew] = (uint16_t)nst;
    P.fc[fnew] = (uint8_t)nc;
    P.fr[fnew] = (uint8_t)nr;
    P.fm0[fnew] = w0;
    P.fm1[fnew] = w1;
    P.fm2[fnew] = w2;
  }
  if (addlid && lane == 0) {
    P.fn[nkeep] = nbr;
    P.fst[nkeep] = (uint16_t)lbase;
    P.fc[nkeep] = (uint8_t)len;
    P.fr[nkeep] = 0;
    P.fm0[nkeep] = A0;
    P.fm1[nkeep] = A1;
    P.fm2[nkeep] = A2;
  }
  const unsigned NL0 = I0 | N0, NL1 = I1 | N1, NL2 = I2 | N2;
  S.live0 = NL0;
  S.live1 = NL1;
  S.live2 = NL2;
  S.nf = nkeep + (addlid ? 1 : 0);
  S.hw = nhw;
  S.cb = dst;
  S.etop = lbase + (addlid ? len : 0);

  // 7. the largest radius over the kept and the new vertices; the mixed
  //    path's bound on the vertices' max norm
  double r2 = 0.0;
  float um = 0.f;
  if (with_gen || C::MIXED) {
#pragma unroll
    for (int w = 0; w < 3; ++w) {
      if (32 * w < nhw) {
        const unsigned Lw = w == 0 ? NL0 : (w == 1 ? NL1 : NL2);
        if ((Lw >> lane) & 1u) {
          const int v = 32 * w + (int)lane;
          r2 = fmax(r2, P.vr2[v]);
          if constexpr (C::MIXED) um = fmaxf(um, P.uin[v]);
        }
      }
    }
  }
  if constexpr (C::MIXED)  // non-negative floats order like their bits
    S.umax = (double)__uint_as_float(__reduce_max_sync(kFull, __float_as_uint(um))) * (1.0 + 0x1p-20);
  if (with_gen) cnt_add(P, kCntKept, (unsigned long long)(__popc(I0) + __popc(I1) + __popc(I2)));
  __syncwarp();
  *r2out = with_gen ? sp_warp_max_nonneg(r2) : 0.0;
  return kClipMod;
}

// volume + centroid (cell_3d_faces.rs:106-205) summed in the reference's
// order -- faces in order, each fanned from its logical first entry -- and
// face_area (:207-254) per face; writes the cell's outputs.
template <class C>
__device__ void finalize_cell(const TessDesc& T, uint32_t i, SparsePoly<C>& P, const SparseState& S) {
  const unsigned lane = lane_id();
  const int nf = S.nf;
  const uint8_t* E = P.ent[S.cb];
  uint8_t* tmap = P.ent[S.cb ^ 1];  // triangle -> face (the spare entry buffer)
  const bool fv = (int)lane < nf;
  int c = 0, st = 0, rot = 0;
  if (fv) {
    c = P.fc[lane];
    st = P.fst[lane];
    rot = P.fr[lane];
  }
  const int t = c >= 3 ? c - 2 : 0;
  const int inc = warp_incl_scan(t);
  const int ntri = __shfl_sync(kFull, inc, 31);
  if (fv) {
    P.xpos[lane] = (uint16_t)(inc - t);
    for (int j = 0; j < t; ++j) tmap[inc - t + j] = (uint8_t)lane;
  }
  __syncwarp();
  double av = 0.0, ax = 0.0, ay = 0.0, az = 0.0;
  for (int b = 0; b < ntri; b += 32) {
    const int tt = b + (int)lane;
    double det = 0.0, dtx = 0.0, dty = 0.0, dtz = 0.0;
    if (tt < ntri) {
      const int f = tmap[tt];
      const int fcn = P.fc[f], fst = P.fst[f], frt = P.fr[f];
      const int j = tt - (int)P.xpos[f] + 1;
      int q1 = j + frt, q2 = j + 1 + frt;
      if (q1 >= fcn) q1 -= fcn;
      if (q2 >= fcn) q2 -= fcn;
      const int i0 = E[fst + frt], i1 = E[fst + q1], i2 = E[fst + q2];
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
  // at most 32 faces: always the cell's own face slots
  int32_t* fnb_out = T.fnb + (size_t)i * T.fout;
  double* far_out = T.farea + (size_t)i * T.fout;
  if (fv) {
    double area = 0.0;
    if (c >= 3) {
      const int p0 = E[st + rot];
      const double p0x = P.vx[p0], p0y = P.vy[p0], p0z = P.vz[p0];
      int q = rot + 1;
      if (q >= c) q -= c;
      for (int j = 1; j < c - 1; ++j) {
        const int q2 = (q + 1 == c) ? 0 : q + 1;
        const int p1 = E[st + q], p2 = E[st + q2];
        const double v1x = P.vx[p1] - p0x, v1y = P.vy[p1] - p0y, v1z = P.vz[p1] - p0z;
        const double v2x = P.vx[p2] - p0x, v2y = P.vy[p2] - p0y, v2z = P.vz[p2] - p0z;
        const double crx = v1y * v2z - v1z * v2y;
        const double cry = v1z * v2x - v1x * v2z;
        const double crz = v1x * v2y - v1y * v2x;
        area += 0.5 * sqrt(crx * crx + cry * cry + crz * crz);
        q = q2;
      }
    }
    fnb_out[lane] = P.fn[lane];
    far_out[lane] = area;
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
    T.nfaces[i] = nf;
    T.nverts[i] = __popc(S.live0) + __popc(S.live1) + __popc(S.live2);
    T.status[i] = kCellOk;
  }
  __syncwarp();
}

// The kernels: persistent warps, each with its polytope in shared memory.
// NOOP: the walk's variant with batched plane tests (compute_cell)
template <class C, int WPB, int MINB, bool NOOP = false>
__global__ void __launch_bounds__(WPB * 32, MINB) k_clip_sparse(const TessDesc T, const WorkList W) {
  extern __shared__ __align__(16) unsigned char smem[];
  SparsePoly<C>* polys = reinterpret_cast<SparsePoly<C>*>(smem);
  clip_worker<C, NOOP>(T, W, polys[threadIdx.x >> 5]);
}

template <class C, int WPB, int MINB>
__global__ void __launch_bounds__(WPB * 32, MINB)
    k_clip_sparse_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess, const WorkList W) {
  extern __shared__ __align__(16) unsigned char smem[];
  SparsePoly<C>* polys = reinterpret_cast<SparsePoly<C>*>(smem);
  clip_worker_batched<C>(descs, tess_off, ntess, W, polys[threadIdx.x >> 5]);
}

}  // namespace vd
