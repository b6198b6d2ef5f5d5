// vd_clip_hub.cuh -- the huge tier's polytope with stable vertex and face
// slots: a modifying clip rewrites only the faces that lose a vertex.
//
// A cell adjacent to thousands of others (the centre of generators on a
// sphere) holds tens of thousands of vertices, and each of its thousands of
// clips cuts away a small cap.  Cell3DFaces::clip_with_scratch
// (cell_3d_faces.rs:288-503) rebuilds the whole polytope on every modifying
// clip, and so does the full-rewrite block layout (vd_clip_block.cuh), so
// such a cell costs clips x size.  Here only the classification visits every
// vertex -- one coalesced pass by the whole block -- and one warp rewrites the
// few faces that lost a vertex:
//  * vertices live in fixed slots; a cut-away vertex's slot is taken by a new
//    intersection vertex or goes on a free list.  Each vertex records its
//    three faces, so the faces a clip touches are found from the vertices it
//    cuts away.
//  * faces live in slots in creation order (the box's six, then one lid per
//    modifying clip) and never move: the live faces in slot order are the
//    reference's face order (survivors in order, the lid last).
//  * a face with no vertex outside the plane comes back from the reference's
//    face walk rotated by one entry (each in->in edge emits its end vertex).
//    Such a face is not touched: its logical first entry follows from the
//    number of modifying clips since it was last written.  A face with an
//    outside vertex is walked from its logical first entry, exactly as the
//    reference walks it, into entries appended to the entry buffer.
// Only the general case is handled, as in the shared-memory slot layout
// (vd_clip_sparse.cuh): every face with a cut-away vertex either keeps no
// vertex or has exactly one in->out and one out->in edge, each crossing edge
// is shared by two such faces, the lid segments form one cycle, and the
// per-clip capacities hold.  Anything else returns kClipOverflow and the cell
// is rebuilt from scratch on the full-rewrite layout, whose results are the
// reference's in every case; both give the same doubles in the same order.
#pragma once
#include "vd_clip_block.cuh"

namespace vd {

struct HubCfg {
  static constexpr int VCAP = 65534;   // vertex slots (16-bit halves of an edge key)
  static constexpr int FCAP = 32767;   // face slots: the box's and one per modifying clip
  static constexpr int ECAP = 196608;  // face entries per entry buffer
  static constexpr int OCAP = 1024;    // vertices one clip cuts away
  static constexpr int KCAP = 512;     // faces of those vertices
  static constexpr int TCAP = 4096;    // edges of those faces
  static constexpr int XCAP = 1024;    // crossing edges per clip (two per rewritten face)
  static constexpr int HCAP = 2048;    // edge-key table (open addressing, at most XCAP / 2 keys)
  static constexpr int RESERVE = 2 * TCAP + XCAP / 2;  // entries one clip may append
  static constexpr int VWORDS = (VCAP + 31) / 32;
  static constexpr int FWORDS = (FCAP + 31) / 32;
  static constexpr int FCHUNK = 512;  // triangles per step of the ordered volume sum
  static constexpr uint32_t kNoKey = 0xFFFFFFFFu;
  static constexpr uint16_t kNone = 0xFFFFu;
};

struct alignas(16) HubPoly {
  // (whole words of slots: the classification reads every slot of a word)
  double vx[32 * HubCfg::VWORDS], vy[32 * HubCfg::VWORDS], vz[32 * HubCfg::VWORDS];
  uint32_t vf[3 * HubCfg::VCAP];  // the three faces of each vertex
  uint32_t freev[HubCfg::VCAP];   // free slots below the high-water mark (a stack)
  int32_t fn[HubCfg::FCAP];       // face neighbour id
  uint32_t fst[HubCfg::FCAP];     // first entry in the current buffer
  uint32_t fc[HubCfg::FCAP];      // entry count (0: the face is gone)
  uint32_t fb[HubCfg::FCAP];      // modifying clips counted when the face was last written:
                                  // logical entry j is ent[fst + (j + M - fb) mod fc]
  uint32_t ftr[HubCfg::FCAP];     // finalize: first triangle of each face
  uint32_t frk[HubCfg::FCAP];     // finalize: output position of each face
  uint32_t ent[2][HubCfg::ECAP];  // face entries (vertex slots); the second buffer for compaction
  // per clip: the new vertices by discovery rank, until every endpoint is read
  double tx[HubCfg::XCAP / 2], ty[HubCfg::XCAP / 2], tz[HubCfg::XCAP / 2];
};

// The block's shared state (dynamic shared memory: about 80 KB)
template <int NW>
struct HubShared {
  BlockShared<NW> blk;            // the walk's staging and the block totals
  unsigned live[HubCfg::VWORDS];  // live vertex slots
  union {
    struct {
      unsigned out[HubCfg::VWORDS];    // per clip: live slots outside the plane
      unsigned claim[HubCfg::FWORDS];  // per clip: faces found from a cut-away vertex
      uint32_t olist[HubCfg::OCAP];    // per clip: the cut-away slots
      // per clip, the faces of the cut-away vertices in slot order (the
      // reference's face order): slot, first entry, count, rotation, first
      // edge of the walk, first new entry, has a crossing
      uint32_t cs[HubCfg::KCAP], cst[HubCfg::KCAP], nst[HubCfg::KCAP];
      uint16_t ccnt[HubCfg::KCAP], crot[HubCfg::KCAP], ctp[HubCfg::KCAP];
      uint8_t ctch[HubCfg::KCAP];
      uint16_t emap[HubCfg::TCAP];     // per clip: the face (rank) of each walked edge
      // per clip: the crossing edges in walk order
      uint32_t xkey[HubCfg::XCAP];     // (min, max) slot pair of the edge
      uint32_t xpos[HubCfg::XCAP];     // entry that receives the intersection vertex
      uint16_t xs[HubCfg::XCAP], xe[HubCfg::XCAP];  // the edge as the face walks it
      uint16_t xf[HubCfg::XCAP];       // rank of the crossing's face
      uint16_t xpart[HubCfg::XCAP];    // the other crossing of the same edge
      uint16_t xid[HubCfg::XCAP];      // slot of the intersection vertex
      uint16_t xr[HubCfg::XCAP];       // discovery rank of the vertex it creates (kNone: reuses)
      uint16_t xhp[HubCfg::XCAP];      // its edge-key table position (kNone: none)
      uint8_t xt[HubCfg::XCAP];        // 1: in->out, 0: out->in
      // edge key -> first crossing, for edges whose second crossing comes in
      // a later round of 32 (emptied after each clip)
      uint32_t hkey[HubCfg::HCAP];
      uint16_t hidx[HubCfg::HCAP];
    } c;
    double tri[4][HubCfg::FCHUNK];     // finalize: one step's per-triangle terms
  } u;
  // per-warp partials of block-wide steps, three steps deep: a step's
  // values are read after its barrier and before the next step's, so a
  // buffer is rewritten (or, for the counter, zeroed) only two steps later
  int pin[3][NW];     // a vertex strictly inside the plane
  double pr2[3][NW];  // largest squared radius of a kept vertex
  int pcnt[3];        // cut-away vertices (a counter)
  int pliv[NW];       // finalize: live vertices
  // polytope state (written by warp 0 before a barrier)
  int nfs, M, hw, nfree, etop, cb, res;
  double r2new;
  unsigned long long pool;
};

// The polytope operations block_walk needs, on the slot layout.  Every thread
// of the block calls each with the same arguments and gets the same result.
template <int NW>
struct HubOps {
  using Cf = HubCfg;
  HubPoly& P;
  HubShared<NW>& H;
  int ser;       // block-wide steps so far (the same in every thread)
  bool isempty;  // an empty clip removed everything

  // Cell3DFaces::new (cell_3d_faces.rs:37-74): the box, faces z-, z+, y-,
  // y+, x-, x+ with ids box_side (bounds/mod.rs:21-22)
  __device__ void init(const Grid& g, double gx, double gy, double gz) {
    const int tid = (int)threadIdx.x, nt = NW * 32;
    for (int k = tid; k < Cf::VWORDS; k += nt) H.live[k] = 0u;
    for (int k = tid; k < Cf::FWORDS; k += nt) H.u.c.claim[k] = 0u;
    for (int k = tid; k < Cf::HCAP; k += nt) H.u.c.hkey[k] = Cf::kNoKey;
    if (tid == 0) H.live[0] = 0xFFu;  // (word 0 was cleared by this thread)
    if (tid < 8) {
      const unsigned hx = (tid == 1 || tid == 2 || tid == 5 || tid == 6);
      const unsigned hy = (tid == 2 || tid == 3 || tid == 6 || tid == 7);
      const unsigned hz = tid >= 4;
      P.vx[tid] = hx ? g.bmax[0] : g.bmin[0];
      P.vy[tid] = hy ? g.bmax[1] : g.bmin[1];
      P.vz[tid] = hz ? g.bmax[2] : g.bmin[2];
      // a corner lies on one face of each axis pair
      P.vf[3 * tid] = hz ? 1u : 0u;
      P.vf[3 * tid + 1] = hy ? 3u : 2u;
      P.vf[3 * tid + 2] = hx ? 5u : 4u;
    }
    // face loops 3210 4567 0154 2376 0473 1265 packed as nibbles, entry = thread
    if (tid < 24) {
      const unsigned long long lo = 0x6732451076540123ull, hi = 0x56213740ull;
      P.ent[0][tid] = (uint32_t)((tid < 16 ? lo >> (4 * tid) : hi >> (4 * (tid - 16))) & 0xFull);
    }
    if (tid < 6) {
      P.fn[tid] = -1 - (2 * (2 - (tid >> 1)) + (tid & 1));
      P.fst[tid] = (uint32_t)(4 * tid);
      P.fc[tid] = 4u;
      P.fb[tid] = 0u;
    }
    if (tid == 0) {
      H.nfs = 6;
      H.M = 0;
      H.hw = 8;
      H.nfree = 0;
      H.etop = 24;
      H.cb = 0;
      H.pcnt[0] = H.pcnt[1] = H.pcnt[2] = 0;
    }
    ser = 0;
    isempty = false;
    __syncthreads();
  }

  __device__ bool empty() const { return isempty; }

  // max_radius_sq (cell_3d_faces.rs:271-286): the largest |v - g|^2 over
  // the live vertices (a maximum does not depend on the order it is taken in)
  __device__ double max_radius(double gx, double gy, double gz) {
    const unsigned lane = lane_id();
    const int w = (int)(threadIdx.x >> 5);
    const int b = ser % 3;
    ++ser;
    if (threadIdx.x == 0) H.pcnt[(b + 1) % 3] = 0;
    const int nwd = (H.hw + 31) >> 5;
    double m = 0.0;
    for (int k = w; k < nwd; k += NW) {
      if ((H.live[k] >> lane) & 1u) {
        const int v = 32 * k + (int)lane;
        const double dx = P.vx[v] - gx, dy = P.vy[v] - gy, dz = P.vz[v] - gz;
        m = fmax(m, dx * dx + dy * dy + dz * dz);
      }
    }
    m = sp_warp_max_nonneg(m);
    if (lane == 0) H.pr2[b][w] = m;
    __syncthreads();
    return sp_warp_max_nonneg((int)lane < NW ? H.pr2[b][lane] : 0.0);
  }

  // the live faces' entries, each face in logical order from its first
  // entry, packed into the other buffer (the appended entries of rewritten
  // faces are left behind); returns the packed size
  __device__ int compact() {
    const unsigned lane = lane_id();
    const int w = (int)(threadIdx.x >> 5);
    const int nfs = H.nfs, M = H.M, src = H.cb, dst = src ^ 1;
    int lo, hi;
    block_range<NW>(nfs, w, &lo, &hi);
    int tot = 0;
    for (int b = lo; b < hi; b += 32) {
      const int f = b + (int)lane;
      tot += f < hi ? (int)P.fc[f] : 0;
    }
    tot = (int)__reduce_add_sync(kFull, (unsigned)tot);
    if (lane == 0) {
      H.blk.a[w] = tot;
      H.blk.b[w] = 0;
      H.blk.c[w] = -1;
    }
    __syncthreads();
    int pa, pb, pc, ta, tb, tc;
    range_prefix<NW>(H.blk, w, &pa, &pb, &pc, &ta, &tb, &tc);
    int run = pa;
    for (int b = lo; b < hi; b += 32) {
      const int f = b + (int)lane;
      const int c = f < hi ? (int)P.fc[f] : 0;
      const int inc = warp_incl_scan(c);
      const int off = run + inc - c;
      if (c > 0) {
        const uint32_t st = P.fst[f];
        int q = (int)((uint32_t)(M - (int)P.fb[f]) % (uint32_t)c);
        for (int j = 0; j < c; ++j) {
          P.ent[dst][off + j] = P.ent[src][st + q];
          q = (q + 1 == c) ? 0 : q + 1;
        }
        P.fst[f] = (uint32_t)off;
        P.fb[f] = (uint32_t)M;
      }
      run += __shfl_sync(kFull, inc, 31);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      H.cb = dst;
      H.etop = ta;
    }
    return ta;
  }

  // clip_with_scratch (cell_3d_faces.rs:288-503) on the slot layout;
  // *r2out: the largest |v - g|^2 over the new vertex set when with_gen
  __device__ int clip(double px, double py, double pz, double nx, double ny, double nz, int nbr, bool with_gen,
                      double gx, double gy, double gz, double* r2out) {
    const unsigned lane = lane_id();
    const unsigned lt = (1u << lane) - 1u;
    const int w = (int)(threadIdx.x >> 5);
    // 0. room for this clip's entries
    if (H.etop + Cf::RESERVE > Cf::ECAP) {
      const int top = compact();
      if (top + Cf::RESERVE > Cf::ECAP) return kClipOverflow;
    }
    const int b = ser % 3;
    ++ser;
    if (threadIdx.x == 0) H.pcnt[(b + 1) % 3] = 0;

    // 1. signed distances of the live vertices and the 3-band flags
    //    (:302-326), a word of slots per warp at a time, four words' loads
    //    in flight (every slot below the high-water mark is read, a free one
    //    ignored); the cut-away slots listed; the kept vertices' largest radius
    const int nwd = (H.hw + 31) >> 5;
    bool sin = false;
    double r2 = 0.0;
    constexpr int U = 4;
    for (int k0 = w; k0 < nwd; k0 += U * NW) {
      double x[U], y[U], z[U];
      unsigned lw[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = k0 + u * NW;
        lw[u] = 0u;
        x[u] = y[u] = z[u] = 0.0;
        if (k < nwd) {
          const int v = 32 * k + (int)lane;
          lw[u] = H.live[k];
          x[u] = P.vx[v];
          y[u] = P.vy[v];
          z[u] = P.vz[v];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = k0 + u * NW;
        if (k >= nwd) break;
        const int v = 32 * k + (int)lane;
        bool o = false;
        if ((lw[u] >> lane) & 1u) {
          const double d = (x[u] - px) * nx + (y[u] - py) * ny + (z[u] - pz) * nz;
          o = d > kTol;
          sin |= d < -kTol;
          if (!o && with_gen) {
            const double dx = x[u] - gx, dy = y[u] - gy, dz = z[u] - gz;
            r2 = fmax(r2, dx * dx + dy * dy + dz * dz);
          }
        }
        const unsigned om = __ballot_sync(kFull, o);
        if (lane == 0) H.u.c.out[k] = om;
        if (om) {
          int pos = 0;
          if (lane == 0) pos = atomicAdd(&H.pcnt[b], __popc(om));
          pos = __shfl_sync(kFull, pos, 0);
          if (o) {
            const int q = pos + __popc(om & lt);
            if (q < Cf::OCAP) H.u.c.olist[q] = (uint32_t)v;
          }
        }
      }
    }
    const bool wsin = __any_sync(kFull, sin);
    const double wr2 = sp_warp_max_nonneg(r2);
    if (lane == 0) {
      H.pin[b][w] = wsin ? 1 : 0;
      H.pr2[b][w] = wr2;
    }
    __syncthreads();
    const int nout = H.pcnt[b];
    const bool any_sin = __any_sync(kFull, (int)lane < NW && H.pin[b][lane] != 0);
    const double r2k = sp_warp_max_nonneg((int)lane < NW ? H.pr2[b][lane] : 0.0);
    if (nout == 0) {
      *r2out = 0.0;
      return kClipNoop;
    }
    if (!any_sin) {
      isempty = true;
      *r2out = 0.0;
      return kClipEmpty;
    }
    if (nout > Cf::OCAP) return kClipOverflow;
    if (w == 0) {
      const int r = rebuild(nout, px, py, pz, nx, ny, nz, nbr, gx, gy, gz);
      if (lane == 0) H.res = r;
    }
    __syncthreads();
    if (H.res != kClipMod) return kClipOverflow;
    *r2out = with_gen ? fmax(r2k, H.r2new) : 0.0;
    return kClipMod;
  }

  // steps 2-7 of the clip by warp 0, 32 elements at a time: the faces of the
  // cut-away vertices are walked and rewritten, the intersection vertices
  // made, the lid added
  __device__ int rebuild(int nout, double px, double py, double pz, double nx, double ny, double nz, int nbr,
                         double gx, double gy, double gz) {
    auto& S = H.u.c;
    const unsigned lane = lane_id();
    const unsigned lt = (1u << lane) - 1u;
    const int M = H.M, nfs = H.nfs, hw = H.hw, nfree = H.nfree, base = H.etop;
    if (nfs >= Cf::FCAP) return kClipOverflow;
    uint32_t* E = P.ent[H.cb];  // new entries are appended after the live ones

    // 2. the faces of the cut-away vertices, each taken once (a face whose
    //    vertices are all kept is not touched: it comes back rotated)
    int ncand = 0;
    for (int k0 = 0; k0 < nout; k0 += 32) {
      const int k = k0 + (int)lane;
      const bool a = k < nout;
      uint32_t f3[3] = {0u, 0u, 0u};
      if (a) {
        const uint32_t o = S.olist[k];
        f3[0] = P.vf[3 * o];
        f3[1] = P.vf[3 * o + 1];
        f3[2] = P.vf[3 * o + 2];
      }
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        bool mine = false;
        if (a) {
          const unsigned bit = 1u << (f3[j] & 31u);
          mine = !(atomicOr(&S.claim[f3[j] >> 5], bit) & bit);
        }
        const unsigned bm = __ballot_sync(kFull, mine);
        if (mine) {
          const int q = ncand + __popc(bm & lt);
          if (q < Cf::KCAP) S.cs[q] = f3[j];
        }
        ncand += __popc(bm);
      }
    }
    if (ncand > Cf::KCAP) return kClipOverflow;
    __syncwarp();
    // in slot order: ranked by the warp when they fit it, else read off the
    // claim bitmap in order
    if (ncand <= 32) {
      const uint32_t fme = (int)lane < ncand ? S.cs[lane] : 0xFFFFFFFFu;
      int rank = 0;
      for (int q = 0; q < ncand; ++q) rank += __shfl_sync(kFull, fme, q) < fme ? 1 : 0;
      __syncwarp();
      if ((int)lane < ncand) S.cs[rank] = fme;
    } else {
      const int nwf = (nfs + 31) >> 5;
      int run = 0;
      for (int k0 = 0; k0 < nwf; k0 += 32) {
        const int k = k0 + (int)lane;
        unsigned wd = k < nwf ? S.claim[k] : 0u;
        const int cw = __popc(wd);
        const int inc = warp_incl_scan(cw);
        int pos = run + inc - cw;
        while (wd) {
          S.cs[pos++] = 32u * (unsigned)k + (unsigned)(__ffs(wd) - 1);
          wd &= wd - 1u;
        }
        run += __shfl_sync(kFull, inc, 31);
      }
    }
    __syncwarp();
    // each face's count, first entry, rotation and first edge of the walk
    int np = 0;
    for (int j0 = 0; j0 < ncand; j0 += 32) {
      const int j = j0 + (int)lane;
      int c = 0;
      if (j < ncand) {
        const uint32_t f = S.cs[j];
        c = (int)P.fc[f];
        S.cst[j] = P.fst[f];
        S.ccnt[j] = (uint16_t)c;
        S.crot[j] = (uint16_t)(c >= 3 ? (uint32_t)(M - (int)P.fb[f]) % (uint32_t)c : 0u);
      }
      if (__any_sync(kFull, j < ncand && c < 3)) return kClipOverflow;
      const int inc = warp_incl_scan(c);
      if (j < ncand) S.ctp[j] = (uint16_t)min(np + inc - c, Cf::TCAP);
      np += __shfl_sync(kFull, inc, 31);
      if (np > Cf::TCAP) return kClipOverflow;
    }
    __syncwarp();
    for (int j0 = 0; j0 < ncand; j0 += 32) {
      const int j = j0 + (int)lane;
      if (j < ncand) {
        const int t0 = S.ctp[j], c = S.ccnt[j];
        for (int q = 0; q < c; ++q) S.emap[t0 + q] = (uint16_t)j;
      }
    }
    __syncwarp();

    // 3. the faces' edges in walk order (faces in order, each from its
    //    logical first entry) -- the face walk of :369-452: in->in emits the
    //    end, in->out the intersection, out->in the intersection and the end.
    //    The new faces follow one another, so an entry's place is the count
    //    of entries emitted before it.  A face that keeps no vertex emits
    //    nothing.
    int run = base, ncr = 0;
    for (int r0 = 0; r0 < np; r0 += 32) {
      const int i = r0 + (int)lane;
      const bool act = i < np;
      uint32_t sv = 0u, ev = 0u;
      bool si = false, ei = false;
      int rk = 0, ftp = -1;
      if (act) {
        rk = S.emap[i];
        const int fst0 = (int)S.cst[rk], fcn = S.ccnt[rk], frot = S.crot[rk];
        ftp = S.ctp[rk];
        int q = i - ftp + frot;
        if (q >= fcn) q -= fcn;
        const int q2 = (q + 1 == fcn) ? 0 : q + 1;
        sv = E[fst0 + q];
        ev = E[fst0 + q2];
        si = !((S.out[sv >> 5] >> (sv & 31u)) & 1u);
        ei = !((S.out[ev >> 5] >> (ev & 31u)) & 1u);
      }
      const int emit = act ? (si ? 1 : (ei ? 2 : 0)) : 0;
      const int einc = warp_incl_scan(emit);
      const int idx = run + einc - emit;
      if (act && i == ftp) S.nst[rk] = (uint32_t)idx;
      const bool cr = act && si != ei;
      const unsigned cm = __ballot_sync(kFull, cr);
      if (cr) {
        const int g = ncr + __popc(cm & lt);
        if (g < Cf::XCAP) {
          S.xkey[g] = sv < ev ? (sv << 16 | ev) : (ev << 16 | sv);
          S.xs[g] = (uint16_t)sv;
          S.xe[g] = (uint16_t)ev;
          S.xpos[g] = (uint32_t)idx;
          S.xt[g] = si ? 1 : 0;
          S.xf[g] = (uint16_t)rk;
        }
      }
      if (act && ei) E[idx + (si ? 0 : 1)] = ev;
      run += __shfl_sync(kFull, einc, 31);
      ncr += __popc(cm);
    }
    if (ncr > Cf::XCAP || (ncr & 1) || ncr < 6) return kClipOverflow;
    const int ntouch = ncr >> 1;
    for (int j0 = 0; j0 < ncand; j0 += 32)
      if (j0 + (int)lane < ncand) S.ctch[j0 + lane] = 0;
    __syncwarp();
    // each face with a crossing has exactly two, consecutive, of opposite
    // directions; the others emitted nothing
    bool bad = false;
    for (int g0 = 0; g0 < ncr; g0 += 32) {
      const int g = g0 + (int)lane;
      if (g < ncr) {
        const int xf = S.xf[g];
        bad |= xf != (int)S.xf[g ^ 1] || S.xt[g] == S.xt[g ^ 1] || ((g & 1) == 0 && g > 0 && (int)S.xf[g - 1] == xf);
        if ((g & 1) == 0) S.ctch[xf] = 1;
      }
    }
    __syncwarp();
    for (int j0 = 0; j0 < ncand; j0 += 32) {
      const int j = j0 + (int)lane;
      if (j < ncand) {
        const uint32_t nx = j + 1 < ncand ? S.nst[j + 1] : (uint32_t)run;
        bad |= !S.ctch[j] && nx != S.nst[j];
      }
    }
    if (__any_sync(kFull, bad)) return kClipOverflow;

    // 4. intersection vertices: the first of the two crossings of an edge in
    //    walk order creates the vertex from its own walk direction, the other
    //    reuses it (the intersection_map of :391-417 / :422-448).  Crossings
    //    go 32 to a round; an edge's second crossing finds the first in the
    //    same round (match.any) or in the edge-key table.  The new vertices
    //    are computed before any is stored: a new vertex may take the slot of
    //    a cut-away endpoint that a later round still reads.
    int nnew = 0;
    double r2n = 0.0;
    double kx = 0.0, ky = 0.0, kz = 0.0;  // the first round's vertices stay in registers
    for (int g0 = 0; g0 < ncr; g0 += 32) {
      const int g = g0 + (int)lane;
      const bool isx = g < ncr;
      const unsigned key = isx ? S.xkey[g] : (0xFFFF0000u | lane);
      const unsigned mm = __match_any_sync(kFull, key);
      const int grp = __popc(mm);
      int hprev = -1, hpos = -1;
      if (isx && g0 == 0) {
        hpos = (int)((key * 2654435761u) >> 21);  // the table is empty in the first round
      } else if (isx) {
        unsigned h = (key * 2654435761u) >> 21;  // 11 bits: HCAP = 2048
        for (int s = 0; s < Cf::HCAP; ++s) {
          const uint32_t k = S.hkey[h];
          if (k == key) {
            hprev = S.hidx[h];
            break;
          }
          if (k == Cf::kNoKey) {
            hpos = (int)h;
            break;
          }
          h = (h + 1u) & (unsigned)(Cf::HCAP - 1);
        }
      }
      bool ldr = false;
      int part = -1;
      if (isx) {
        if (hprev >= 0) {
          part = hprev;  // the second crossing of an edge begun in an earlier round
          bad |= grp != 1;
        } else if (grp == 2) {
          const int o = __ffs(mm & ~(1u << lane)) - 1;
          part = g0 + o;
          ldr = (int)lane < o;
        } else if (grp == 1) {
          ldr = true;  // its partner comes in a later round (there is none in one round)
          bad |= hpos < 0 || ncr <= 32;
        } else {
          bad = true;
        }
      }
      if (__any_sync(kFull, bad)) return kClipOverflow;
      // enter the edges still waiting for their second crossing (keys of one
      // round are distinct)
      uint16_t hp = Cf::kNone;
      if (isx && hprev < 0 && grp == 1) {
        unsigned h = (unsigned)hpos;
        for (int s = 0; s < Cf::HCAP; ++s) {
          if (atomicCAS(&S.hkey[h], Cf::kNoKey, key) == Cf::kNoKey) {
            S.hidx[h] = (uint16_t)g;
            hp = (uint16_t)h;
            break;
          }
          h = (h + 1u) & (unsigned)(Cf::HCAP - 1);
        }
        bad |= hp == Cf::kNone;
      }
      if (isx) {
        S.xhp[g] = hp;
        S.xpart[g] = part >= 0 ? (uint16_t)part : Cf::kNone;
        if (hprev >= 0) S.xpart[hprev] = (uint16_t)g;
      }
      // the new vertex of discovery rank r takes the r-th cut-away slot, then
      // the free list, then a slot above the high-water mark
      const unsigned lm = __ballot_sync(kFull, ldr);
      uint16_t xr = Cf::kNone;
      if (ldr && nnew + __popc(lm & lt) >= Cf::XCAP / 2) bad = true;  // unpaired crossings
      if (ldr && !bad) {
        const int r = nnew + __popc(lm & lt);
        const int slot = r < nout ? (int)S.olist[r]
                                  : (r - nout < nfree ? (int)P.freev[nfree - 1 - (r - nout)] : hw + (r - nout - nfree));
        bad |= slot >= Cf::VCAP;
        const uint32_t s = S.xs[g], e = S.xe[g];
        const double ax = P.vx[s], ay = P.vy[s], az = P.vz[s];
        const double bx = P.vx[e], by = P.vy[e], bz = P.vz[e];
        // the classification's distances, recomputed with the same expression
        const double ds = (ax - px) * nx + (ay - py) * ny + (az - pz) * nz;
        const double de = (bx - px) * nx + (by - py) * ny + (bz - pz) * nz;
        const double t = clamp01(ds / (ds - de));
        const double ix = ax + t * (bx - ax), iy = ay + t * (by - ay), iz = az + t * (bz - az);
        if (g0 == 0) {
          kx = ix;
          ky = iy;
          kz = iz;
        } else {
          P.tx[r] = ix;
          P.ty[r] = iy;
          P.tz[r] = iz;
        }
        const double dx = ix - gx, dy = iy - gy, dz = iz - gz;
        r2n = fmax(r2n, dx * dx + dy * dy + dz * dz);
        S.xid[g] = (uint16_t)min(slot, Cf::VCAP);
        xr = (uint16_t)r;
      }
      if (isx) S.xr[g] = xr;
      nnew += __popc(lm);
      __syncwarp();
      if (isx && !ldr) S.xid[g] = S.xid[hprev >= 0 ? hprev : part];
      __syncwarp();
    }
    // the edges entered in the table leave it; every crossing has a partner
    // walked the other way
    for (int g0 = 0; g0 < ncr; g0 += 32) {
      const int g = g0 + (int)lane;
      if (g < ncr) {
        if (S.xhp[g] != Cf::kNone) S.hkey[S.xhp[g]] = Cf::kNoKey;
        const int pt = S.xpart[g];
        bad |= pt == Cf::kNone || S.xt[pt] == S.xt[g];
      }
    }
    if (__any_sync(kFull, bad)) return kClipOverflow;
    const int grow = max(0, nnew - nout - nfree);
    __syncwarp();
    // the new vertices stored, each with its faces: the two across its edge
    // and the lid; every intersection entry written
    for (int g0 = 0; g0 < ncr; g0 += 32) {
      const int g = g0 + (int)lane;
      if (g < ncr) {
        const int slot = S.xid[g];
        const int r = S.xr[g];
        if (r != Cf::kNone) {
          P.vx[slot] = g0 == 0 ? kx : P.tx[r];
          P.vy[slot] = g0 == 0 ? ky : P.ty[r];
          P.vz[slot] = g0 == 0 ? kz : P.tz[r];
          P.vf[3 * slot] = S.cs[S.xf[g]];
          P.vf[3 * slot + 1] = S.cs[S.xf[S.xpart[g]]];
          P.vf[3 * slot + 2] = (uint32_t)nfs;
        }
        E[S.xpos[g]] = (uint32_t)slot;
      }
    }

    // 5. the lid (:470-495): touched face k gives the segment (X of its
    //    out->in crossing, X of its in->out crossing); the segment after k
    //    is the face of its in->out crossing's partner.  The chain from
    //    segment 0 must take every segment.
    const int lbase = run;
    if (ntouch <= 32) {  // ranked by pointer jumping
      const bool sact = (int)lane < ntouch;
      unsigned a = 0u, succ = lane;
      if (sact) {
        const bool io0 = S.xt[2 * lane] != 0;  // crossing 2k is the in->out one
        a = S.xid[io0 ? 2 * lane + 1 : 2 * lane];
        succ = (unsigned)(S.xpart[io0 ? 2 * lane : 2 * lane + 1] >> 1);
      }
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
      if (term < 0 || d0 + 1 != ntouch || __any_sync(kFull, sact && (nxt != term || dd < 0 || dd > d0)))
        return kClipOverflow;
      if (sact) E[lbase + d0 - dd] = a;
    } else {  // followed by one lane
      int ok = 0;
      if (lane == 0) {
        int k = 0, pos = 0;
        do {
          const bool io0 = S.xt[2 * k] != 0;
          if (pos < ntouch) E[lbase + pos] = S.xid[io0 ? 2 * k + 1 : 2 * k];
          ++pos;
          k = S.xpart[io0 ? 2 * k : 2 * k + 1] >> 1;
        } while (k != 0 && pos <= ntouch);
        ok = (k == 0 && pos == ntouch) ? 1 : 0;
      }
      if (!__shfl_sync(kFull, ok, 0)) return kClipOverflow;
    }

    // 6. the face table: rewritten faces point at their new entries, faces
    //    that kept no vertex are gone, the lid takes the next slot
    for (int j0 = 0; j0 < ncand; j0 += 32) {
      const int j = j0 + (int)lane;
      if (j < ncand) {
        const uint32_t f = S.cs[j];
        if (S.ctch[j]) {
          const uint32_t nx = j + 1 < ncand ? S.nst[j + 1] : (uint32_t)run;
          P.fst[f] = S.nst[j];
          P.fc[f] = nx - S.nst[j];
          P.fb[f] = (uint32_t)(M + 1);
        } else {
          P.fc[f] = 0u;
        }
        atomicAnd(&S.claim[f >> 5], ~(1u << (f & 31u)));
      }
    }
    if (lane == 0) {
      P.fn[nfs] = nbr;
      P.fst[nfs] = (uint32_t)lbase;
      P.fc[nfs] = (uint32_t)ntouch;
      P.fb[nfs] = (uint32_t)(M + 1);
    }
    // 7. live slots: the cut-away ones leave, the new ones join; cut-away
    //    slots that no new vertex took go on the free list
    for (int k = (int)lane; k < nout; k += 32) {
      const uint32_t o = S.olist[k];
      atomicAnd(&H.live[o >> 5], ~(1u << (o & 31u)));
    }
    __syncwarp();
    for (int g0 = 0; g0 < ncr; g0 += 32) {
      const int g = g0 + (int)lane;
      if (g < ncr && S.xr[g] != Cf::kNone) {
        const unsigned slot = S.xid[g];
        atomicOr(&H.live[slot >> 5], 1u << (slot & 31u));
      }
    }
    for (int k = nnew + (int)lane; k < nout; k += 32) P.freev[nfree + (k - nnew)] = S.olist[k];
    const int popd = min(max(nnew - nout, 0), nfree);
    r2n = sp_warp_max_nonneg(r2n);
    if (lane == 0) {
      H.nfs = nfs + 1;
      H.M = M + 1;
      H.hw = hw + grow;
      H.nfree = nfree - popd + max(nout - nnew, 0);
      H.etop = lbase + ntouch;
      H.r2new = r2n;
    }
    return kClipMod;
  }
};

// volume + centroid (cell_3d_faces.rs:106-205) summed in the reference's
// order -- live faces in slot order, each fanned from its logical first
// entry -- and face_area (:207-254) per face, by the whole block; writes the
// cell's outputs.  The per-triangle terms are computed in parallel, a step
// of FCHUNK at a time, and warp 0 adds them in order.
template <int NW>
__device__ void finalize_hub(const TessDesc& T, uint32_t i, HubPoly& P, HubShared<NW>& H, bool isempty) {
  using Cf = HubCfg;
  const unsigned lane = lane_id();
  const int w = (int)(threadIdx.x >> 5);
  const int tid = (int)threadIdx.x, nt = NW * 32;
  if (isempty) {
    if (tid == 0) {
      T.vol[i] = 0.0;
      T.cen[3 * (size_t)i] = 0.0;
      T.cen[3 * (size_t)i + 1] = 0.0;
      T.cen[3 * (size_t)i + 2] = 0.0;
      T.nfaces[i] = 0;
      T.nverts[i] = 0;
      T.status[i] = kCellOk;
    }
    return;
  }
  const int nfs = H.nfs, M = H.M, cb = H.cb;
  const int nwd = (H.hw + 31) >> 5;
  const uint32_t* E = P.ent[cb];
  uint32_t* tmap = P.ent[cb ^ 1];  // triangle -> face (the spare entry buffer)
  // live faces, triangles and vertices per range
  int lo, hi;
  block_range<NW>(nfs, w, &lo, &hi);
  int nl = 0, ntr = 0, nlv = 0;
  for (int b = lo; b < hi; b += 32) {
    const int f = b + (int)lane;
    const int c = f < hi ? (int)P.fc[f] : 0;
    nl += c > 0 ? 1 : 0;
    ntr += c >= 3 ? c - 2 : 0;
  }
  for (int k = w * 32 + (int)lane; k < nwd; k += nt) nlv += __popc(H.live[k]);
  nl = (int)__reduce_add_sync(kFull, (unsigned)nl);
  ntr = (int)__reduce_add_sync(kFull, (unsigned)ntr);
  nlv = (int)__reduce_add_sync(kFull, (unsigned)nlv);
  if (lane == 0) {
    H.blk.a[w] = nl;
    H.blk.b[w] = ntr;
    H.blk.c[w] = -1;
    H.pliv[w] = nlv;
  }
  __syncthreads();
  int pa, pb, pc, nf, ntri, tc;
  range_prefix<NW>(H.blk, w, &pa, &pb, &pc, &nf, &ntri, &tc);
  const int nverts = (int)__reduce_add_sync(kFull, (int)lane < NW ? (unsigned)H.pliv[lane] : 0u);
  // each live face's output position and first triangle; triangle -> face
  int rf = pa, rt = pb;
  for (int b = lo; b < hi; b += 32) {
    const int f = b + (int)lane;
    const int c = f < hi ? (int)P.fc[f] : 0;
    const int lv = c > 0 ? 1 : 0;
    const int t = c >= 3 ? c - 2 : 0;
    const int incf = warp_incl_scan(lv), inct = warp_incl_scan(t);
    if (lv) {
      const int t0 = rt + inct - t;
      P.frk[f] = (uint32_t)(rf + incf - 1);
      P.ftr[f] = (uint32_t)t0;
      for (int j = 0; j < t; ++j) tmap[t0 + j] = (uint32_t)f;
    }
    rf += __shfl_sync(kFull, incf, 31);
    rt += __shfl_sync(kFull, inct, 31);
  }
  if (tid == 0) {
    unsigned long long off = ~0ull;
    if (nf > T.fout && T.pool_cursor) {
      const unsigned long long o = atomicAdd(T.pool_cursor, (unsigned long long)nf);
      if ((long long)(o + nf) <= T.pool_cap) off = o;
    }
    H.pool = off;
  }
  __syncthreads();
  const int fout = T.fout;
  int32_t* fnb_out = nullptr;
  double* far_out = nullptr;
  if (nf <= fout) {
    fnb_out = T.fnb + (size_t)i * fout;
    far_out = T.farea + (size_t)i * fout;
  } else if (H.pool != ~0ull) {
    fnb_out = T.pool_fnb + H.pool;
    far_out = T.pool_farea + H.pool;
    if (tid == 0) T.pool_off[i] = (long long)H.pool;
  }
  // face areas, a face per thread
  for (int f = tid; f < nfs; f += nt) {
    const int c = (int)P.fc[f];
    if (c == 0) continue;
    const int st = (int)P.fst[f];
    const int rot = (int)((uint32_t)(M - (int)P.fb[f]) % (uint32_t)c);
    double area = 0.0;
    const uint32_t p0 = E[st + rot];
    const double p0x = P.vx[p0], p0y = P.vy[p0], p0z = P.vz[p0];
    int q = rot + 1;
    if (q >= c) q -= c;
    for (int j = 1; j < c - 1; ++j) {
      const int q2 = (q + 1 == c) ? 0 : q + 1;
      const uint32_t p1 = E[st + q], p2 = E[st + q2];
      const double v1x = P.vx[p1] - p0x, v1y = P.vy[p1] - p0y, v1z = P.vz[p1] - p0z;
      const double v2x = P.vx[p2] - p0x, v2y = P.vy[p2] - p0y, v2z = P.vz[p2] - p0z;
      const double crx = v1y * v2z - v1z * v2y;
      const double cry = v1z * v2x - v1x * v2z;
      const double crz = v1x * v2y - v1y * v2x;
      area += 0.5 * sqrt(crx * crx + cry * cry + crz * crz);
      q = q2;
    }
    if (fnb_out) {
      const uint32_t r = P.frk[f];
      fnb_out[r] = P.fn[f];
      far_out[r] = area;
    }
  }
  // the ordered sums over all triangles
  double av = 0.0, ax = 0.0, ay = 0.0, az = 0.0;
  for (int t0 = 0; t0 < ntri; t0 += Cf::FCHUNK) {
    for (int tt = tid; tt < Cf::FCHUNK; tt += nt) {
      const int t = t0 + tt;
      double det = 0.0, dtx = 0.0, dty = 0.0, dtz = 0.0;
      if (t < ntri) {
        const uint32_t f = tmap[t];
        const int c = (int)P.fc[f], st = (int)P.fst[f];
        const int rot = (int)((uint32_t)(M - (int)P.fb[f]) % (uint32_t)c);
        const int j = t - (int)P.ftr[f] + 1;
        int q1 = j + rot, q2 = j + 1 + rot;
        if (q1 >= c) q1 -= c;
        if (q2 >= c) q2 -= c;
        const uint32_t i0 = E[st + rot], i1 = E[st + q1], i2 = E[st + q2];
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
      H.u.tri[0][tt] = det;
      H.u.tri[1][tt] = dtx;
      H.u.tri[2][tt] = dty;
      H.u.tri[3][tt] = dtz;
    }
    __syncthreads();
    if (w == 0) {
      const int n = min(Cf::FCHUNK, ntri - t0);
      for (int j = 0; j < n; ++j) {
        av += H.u.tri[0][j];
        ax += H.u.tri[1][j];
        ay += H.u.tri[2][j];
        az += H.u.tri[3][j];
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
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
    const bool ok = fnb_out != nullptr || nf == 0;
    T.nfaces[i] = ok ? nf : -1;
    T.nverts[i] = nverts;
    T.status[i] = ok ? kCellOk : kCellHardFail;
  }
}

// one cell by the block: on the slot layout unless its polytope is exported
// (which needs the reference's vertex order), on the full-rewrite layout when
// the slot layout hands the cell back; returns the cell's status, with its
// outputs written when that is kCellOk
template <class C, int NW>
__device__ int huge_cell(const TessDesc& T, uint32_t cell, WarpPoly<C>& P, HubShared<NW>& H, const WorkList& W) {
  static_assert(sizeof(HubPoly) <= sizeof(WarpPoly<C>), "the slot layout lives in the block's polytope memory");
  const bool exported = W.ex_verts != nullptr;
  if (!exported) {
    HubOps<NW> X{*reinterpret_cast<HubPoly*>(&P), H, 0, false};
    const int st = block_walk<NW>(T, cell, H.blk, X);
    __syncthreads();
    if (st == kCellOk) finalize_hub<NW>(T, cell, X.P, H, X.isempty);
    if (st != kCellOverflow) return st;
  }
  PolyState S;
  const int st = compute_cell_block<C, NW>(T, cell, P, H.blk, S);
  __syncthreads();
  if (st == kCellOk && (threadIdx.x >> 5) == 0) {
    finalize_cell<C>(T, cell, P, S);
    if (exported) export_cell<C>(W, P, S);
  }
  return st;
}

// persistent blocks over the listed cells, one cell per block at a time; the
// block's polytope lives in global memory
template <class C, int NW>
__global__ void __launch_bounds__(NW * 32)
    k_clip_huge_block(const TessDesc T, const WorkList W, WarpPoly<C>* polys) {
  extern __shared__ __align__(16) unsigned char hub_smem[];
  HubShared<NW>& H = *reinterpret_cast<HubShared<NW>*>(hub_smem);
  WarpPoly<C>& P = polys[blockIdx.x];
  while (true) {
    if (threadIdx.x == 0) H.blk.idx = atomicAdd(W.cursor, 1u);
    __syncthreads();
    const unsigned idx = H.blk.idx;
    __syncthreads();
    if (idx >= W.nitems) break;
    const uint32_t cell = W.items ? W.items[idx] : (uint32_t)T.sorted[idx].id;
    const int st = huge_cell<C, NW>(T, cell, P, H, W);
    if (st != kCellOk && threadIdx.x == 0) {
      T.status[cell] = (uint8_t)st;
      if (st == kCellOverflow && W.ovf_list) W.ovf_list[atomicAdd(W.ovf_count, 1u)] = cell;
      if (st == kCellTable && W.tab_list) W.tab_list[atomicAdd(W.tab_count, 1u)] = cell;
    }
    __syncthreads();
  }
}

// the same over a batch's work list: items are global positions in the
// concatenated bin-ordered generators (clip_worker_batched)
template <class C, int NW>
__global__ void __launch_bounds__(NW * 32)
    k_clip_huge_block_batched(const TessDesc* descs, const uint32_t* tess_off, int ntess, const WorkList W,
                              WarpPoly<C>* polys) {
  extern __shared__ __align__(16) unsigned char hub_smem[];
  HubShared<NW>& H = *reinterpret_cast<HubShared<NW>*>(hub_smem);
  WarpPoly<C>& P = polys[blockIdx.x];
  const uint32_t nitems = W.nitems_dev ? *W.nitems_dev : W.nitems;
  while (true) {
    if (threadIdx.x == 0) H.blk.idx = atomicAdd(W.cursor, 1u);
    __syncthreads();
    const unsigned idx = H.blk.idx;
    __syncthreads();
    if (idx >= nitems) break;
    const uint32_t item = W.items ? W.items[idx] : idx;
    const int t = find_tess(tess_off, ntess, item);
    const TessDesc& T = descs[t];
    const uint32_t cell = (uint32_t)T.sorted[item].id;
    const int st = huge_cell<C, NW>(T, cell, P, H, W);
    if (st != kCellOk && threadIdx.x == 0) {
      T.status[cell] = (uint8_t)st;
      if (st == kCellOverflow && W.ovf_list) W.ovf_list[atomicAdd(W.ovf_count, 1u)] = item;
      if (st == kCellTable) {
        if (W.tab_list) W.tab_list[atomicAdd(W.tab_count, 1u)] = item;
        if (W.tess_flags) atomicOr(&W.tess_flags[t], 1u);
      }
    }
    __syncthreads();
  }
}


}  // namespace vd
