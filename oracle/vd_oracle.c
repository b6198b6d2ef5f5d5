/*
 * vd_oracle.c -- CPU oracle for the 3D tessellation path (TEST INFRASTRUCTURE).
 *
 * A plain-C restatement of the reference crate `voronoid`:
 *   src/tessellation.rs        set_generators :43-67, add_wall/prune :175-200,
 *                              calculate :213-230, compute_cell :414-475,
 *                              relax :482-495
 *   src/algorithm/algo_3d_grid.rs  new + search order :47-95,
 *                              get_bin_index :98-107, set_generators :111-130,
 *                              visit_neighbors :145-202
 *   src/cell/cell_3d_faces.rs  new :37-74, volume :106-143, centroid :145-205,
 *                              face_area :207-254, max_radius_sq :271-286,
 *                              clip_with_scratch :288-503
 *   src/wall/wall_3d.rs        PlaneGeometry :23-46, SphereGeometry :72-101,
 *                              CylinderGeometry :107-174, ConeGeometry :177-262,
 *                              TorusGeometry :265-365, ConvexPolyhedronGeometry :462-708
 *   src/wall/mod.rs            WALL_ID_MAX and the id check :8,24-27
 *   src/bounds/mod.rs          box_side :21-22
 *
 * Arithmetic is written in the reference's evaluation order and must be
 * compiled with -ffp-contract=off (Rust never fuses a multiply and an add),
 * so that every double matches what the reference computes.
 *
 * Only the tests, the smoke check and the CPU-baseline leg of the benchmark
 * use this file, as a checker; the product never links it.
 */
#include "vd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define VDO_TOL 1e-9 /* cell_3d_faces.rs:310-315,346,383-384 */
#define VDO_WALL_ID_MAX (-1000)
#define VDO_MAX_WALLS 64
#define U16_NONE 0xFFFFu

/* ------------------------------------------------------------------ */
/* growable arrays                                                      */
/* ------------------------------------------------------------------ */
static void* grow(void* p, size_t* cap, size_t need, size_t elem) {
  if (need <= *cap) return p;
  size_t nc = *cap ? *cap : 16;
  while (nc < need) nc *= 2;
  void* q = realloc(p, nc * elem);
  if (!q) abort();
  *cap = nc;
  return q;
}
#define GROW(arr, cap, need) ((arr) = grow((arr), &(cap), (need), sizeof(*(arr))))

/* ------------------------------------------------------------------ */
/* cell (cell_3d_faces.rs:24-34)                                        */
/* ------------------------------------------------------------------ */
struct vdo_cell {
  size_t id;
  double* v;     size_t nv, cap_v;  /* nv vertices, 3 doubles each */
  uint8_t* fc;   size_t nf, cap_fc; /* face counts, u8 as in the reference */
  int32_t* fn;   size_t cap_fn;     /* face neighbours */
  uint16_t* fi;  size_t nh, cap_fi; /* flattened face indices, u16 */
};

typedef struct {
  double* v;      size_t nv, cap_v;
  uint8_t* fc;    size_t nf, cap_fc;
  int32_t* fn;    size_t cap_fn;
  uint16_t* fi;   size_t nh, cap_fi;
  double* dists;  size_t cap_d;
  uint8_t* is_int; size_t cap_ii;
  int32_t* o2n;   size_t cap_o2n;     /* Option<u16>: -1 = None */
  uint32_t* ikey; uint16_t* iid; size_t ni, cap_ik, cap_iid;
  uint16_t* lseg; size_t nseg, cap_ls; /* pairs */
  uint16_t* fbuf; size_t nfb, cap_fb;
  uint16_t* lbuf; size_t nlb, cap_lb;
  uint16_t* lmap; size_t cap_lm;
} scratch_t;

static void scratch_free(scratch_t* s) {
  free(s->v); free(s->fc); free(s->fn); free(s->fi); free(s->dists);
  free(s->is_int); free(s->o2n); free(s->ikey); free(s->iid); free(s->lseg);
  free(s->fbuf); free(s->lbuf); free(s->lmap);
  memset(s, 0, sizeof(*s));
}

/* box_side (bounds/mod.rs:21-22): x- -1, x+ -2, y- -3, y+ -4, z- -5, z+ -6 */
static int32_t box_side(int axis, int is_max) { return -1 - (axis * 2 + (is_max ? 1 : 0)); }

/* Cell3DFaces::new (cell_3d_faces.rs:37-74) */
static void cell_init_box(vdo_cell* c, size_t id, const double* mn, const double* mx) {
  static const uint16_t idx[24] = {3, 2, 1, 0, 4, 5, 6, 7, 0, 1, 5, 4,
                                   2, 3, 7, 6, 0, 4, 7, 3, 1, 2, 6, 5};
  const double vv[24] = {mn[0], mn[1], mn[2], mx[0], mn[1], mn[2], mx[0], mx[1], mn[2],
                         mn[0], mx[1], mn[2], mn[0], mn[1], mx[2], mx[0], mn[1], mx[2],
                         mx[0], mx[1], mx[2], mn[0], mx[1], mx[2]};
  c->id = id;
  GROW(c->v, c->cap_v, 24);
  memcpy(c->v, vv, sizeof(vv));
  c->nv = 8;
  GROW(c->fc, c->cap_fc, 6);
  GROW(c->fn, c->cap_fn, 6);
  for (int f = 0; f < 6; ++f) c->fc[f] = 4;
  c->fn[0] = box_side(2, 0); c->fn[1] = box_side(2, 1);
  c->fn[2] = box_side(1, 0); c->fn[3] = box_side(1, 1);
  c->fn[4] = box_side(0, 0); c->fn[5] = box_side(0, 1);
  c->nf = 6;
  GROW(c->fi, c->cap_fi, 24);
  memcpy(c->fi, idx, sizeof(idx));
  c->nh = 24;
}

/* max_radius_sq (cell_3d_faces.rs:271-286) */
static double cell_max_radius_sq(const vdo_cell* c, const double* g) {
  double m = 0.0;
  for (size_t k = 0; k < c->nv; ++k) {
    double dx = c->v[3 * k] - g[0];
    double dy = c->v[3 * k + 1] - g[1];
    double dz = c->v[3 * k + 2] - g[2];
    double d2 = dx * dx + dy * dy + dz * dz;
    if (d2 > m) m = d2;
  }
  return m;
}

static inline double clamp01(double x) {
  /* f64::clamp(0.0, 1.0): NaN passes through */
  if (x < 0.0) return 0.0;
  if (x > 1.0) return 1.0;
  return x;
}

/* intersection lookup/creation shared by both crossing cases
 * (cell_3d_faces.rs:391-417 and :422-448) */
static uint16_t intersect(const vdo_cell* c, scratch_t* s, size_t is, size_t ie,
                          const double* g, double* max_d2, uint64_t* cnt) {
  uint32_t key = is < ie ? ((uint32_t)is << 16 | (uint32_t)ie) : ((uint32_t)ie << 16 | (uint32_t)is);
  for (size_t k = 0; k < s->ni; ++k)
    if (s->ikey[k] == key) return s->iid[k];
  double ds = s->dists[is], de = s->dists[ie];
  double t = clamp01(ds / (ds - de));
  double ax = c->v[is * 3], ay = c->v[is * 3 + 1], az = c->v[is * 3 + 2];
  double bx = c->v[ie * 3], by = c->v[ie * 3 + 1], bz = c->v[ie * 3 + 2];
  uint16_t nid = (uint16_t)s->nv;
  double nx = ax + t * (bx - ax);
  double ny = ay + t * (by - ay);
  double nz = az + t * (bz - az);
  GROW(s->v, s->cap_v, 3 * (s->nv + 1));
  s->v[3 * s->nv] = nx; s->v[3 * s->nv + 1] = ny; s->v[3 * s->nv + 2] = nz;
  s->nv++;
  if (g) {
    double dx = nx - g[0], dy = ny - g[1], dz = nz - g[2];
    double d2 = dx * dx + dy * dy + dz * dz;
    if (d2 > *max_d2) *max_d2 = d2;
  }
  GROW(s->is_int, s->cap_ii, s->nv);
  s->is_int[s->nv - 1] = 1;
  GROW(s->ikey, s->cap_ik, s->ni + 1);
  GROW(s->iid, s->cap_iid, s->ni + 1);
  s->ikey[s->ni] = key; s->iid[s->ni] = nid; s->ni++;
  if (cnt) cnt[VDO_CNT_INTERSECTIONS]++;
  return nid;
}

static inline void fbuf_push(scratch_t* s, uint16_t x) {
  GROW(s->fbuf, s->cap_fb, s->nfb + 1);
  s->fbuf[s->nfb++] = x;
}

/* clip_with_scratch (cell_3d_faces.rs:288-503).  Returns modified; *r2 gets
 * the new max radius over the new vertex set when g != NULL, else 0. */
static int cell_clip(vdo_cell* c, const double* p, const double* n, int32_t nbr,
                     scratch_t* s, const double* g, double* r2, uint64_t* cnt) {
  const double px = p[0], py = p[1], pz = p[2];
  const double nx = n[0], ny = n[1], nz = n[2];
  const size_t nv = c->nv;
  int all_in = 1, all_out = 1;
  *r2 = 0.0;
  if (cnt) { cnt[VDO_CNT_CLIPS]++; cnt[VDO_CNT_CLASSIFIED] += nv; }
  GROW(s->dists, s->cap_d, nv);
  /* 1. distances (:302-315) */
  for (size_t i = 0; i < nv; ++i) {
    double vx = c->v[3 * i], vy = c->v[3 * i + 1], vz = c->v[3 * i + 2];
    double d = (vx - px) * nx + (vy - py) * ny + (vz - pz) * nz;
    s->dists[i] = d;
    if (d > VDO_TOL) all_in = 0;
    else if (d < -VDO_TOL) all_out = 0;
  }
  if (all_in) return 0;
  if (all_out) {
    c->nv = 0; c->nf = 0; c->nh = 0;
    return 1;
  }
  if (cnt) cnt[VDO_CNT_MODIFYING]++;
  /* 2. new structures (:328-340) */
  s->nv = 0; s->nf = 0; s->nh = 0; s->ni = 0; s->nseg = 0;
  GROW(s->o2n, s->cap_o2n, nv);
  for (size_t i = 0; i < nv; ++i) s->o2n[i] = -1;
  double max_d2 = 0.0;
  /* keep inside vertices in order (:344-362) */
  for (size_t i = 0; i < nv; ++i) {
    if (s->dists[i] <= VDO_TOL) {
      uint16_t nid = (uint16_t)s->nv;
      GROW(s->v, s->cap_v, 3 * (s->nv + 1));
      s->v[3 * s->nv] = c->v[3 * i];
      s->v[3 * s->nv + 1] = c->v[3 * i + 1];
      s->v[3 * s->nv + 2] = c->v[3 * i + 2];
      s->nv++;
      s->o2n[i] = nid;
      GROW(s->is_int, s->cap_ii, s->nv);
      s->is_int[s->nv - 1] = 0;
      if (g) {
        double dx = c->v[3 * i] - g[0];
        double dy = c->v[3 * i + 1] - g[1];
        double dz = c->v[3 * i + 2] - g[2];
        double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 > max_d2) max_d2 = d2;
        if (cnt) cnt[VDO_CNT_KEPT]++;
      }
    }
  }
  /* 3. clip each face (:369-468) */
  size_t off = 0;
  for (size_t f = 0; f < c->nf; ++f) {
    size_t count = c->fc[f];
    int32_t fnb = c->fn[f];
    const uint16_t* cur = &c->fi[off];
    off += count;
    s->nfb = 0;
    for (size_t i = 0; i < count; ++i) {
      size_t is = cur[i], ie = cur[(i + 1) % count];
      double ds = s->dists[is], de = s->dists[ie];
      int s_in = ds <= VDO_TOL, e_in = de <= VDO_TOL;
      if (s_in) {
        if (e_in) {
          if (s->o2n[ie] >= 0) fbuf_push(s, (uint16_t)s->o2n[ie]);
        } else {
          fbuf_push(s, intersect(c, s, is, ie, g, &max_d2, cnt));
        }
      } else if (e_in) {
        fbuf_push(s, intersect(c, s, is, ie, g, &max_d2, cnt));
        if (s->o2n[ie] >= 0) fbuf_push(s, (uint16_t)s->o2n[ie]);
      }
    }
    if (s->nfb >= 3) {
      GROW(s->fc, s->cap_fc, s->nf + 1);
      GROW(s->fn, s->cap_fn, s->nf + 1);
      s->fc[s->nf] = (uint8_t)s->nfb;
      s->fn[s->nf] = fnb;
      s->nf++;
      for (size_t i = 0; i < s->nfb; ++i) {
        uint16_t u = s->fbuf[i], v = s->fbuf[(i + 1) % s->nfb];
        if (s->is_int[u] && s->is_int[v]) {
          GROW(s->lseg, s->cap_ls, 2 * (s->nseg + 1));
          s->lseg[2 * s->nseg] = v;
          s->lseg[2 * s->nseg + 1] = u;
          s->nseg++;
        }
      }
      GROW(s->fi, s->cap_fi, s->nh + s->nfb);
      memcpy(&s->fi[s->nh], s->fbuf, s->nfb * sizeof(uint16_t));
      s->nh += s->nfb;
    }
  }
  /* 4. lid face (:470-495) */
  if (s->nseg > 0) {
    s->nlb = 0;
    GROW(s->lmap, s->cap_lm, s->nv);
    for (size_t k = 0; k < s->nv; ++k) s->lmap[k] = U16_NONE;
    for (size_t k = 0; k < s->nseg; ++k) s->lmap[s->lseg[2 * k]] = s->lseg[2 * k + 1];
    uint16_t start = s->lseg[0], next = s->lseg[1];
    GROW(s->lbuf, s->cap_lb, s->nlb + 1);
    s->lbuf[s->nlb++] = start;
    uint16_t curv = next;
    while (curv != start && s->nlb <= s->nseg) {
      GROW(s->lbuf, s->cap_lb, s->nlb + 1);
      s->lbuf[s->nlb++] = curv;
      curv = s->lmap[curv];
      if (curv == U16_NONE) break;
    }
    if (s->nlb >= 3) {
      GROW(s->fc, s->cap_fc, s->nf + 1);
      GROW(s->fn, s->cap_fn, s->nf + 1);
      s->fc[s->nf] = (uint8_t)s->nlb;
      s->fn[s->nf] = nbr;
      s->nf++;
      GROW(s->fi, s->cap_fi, s->nh + s->nlb);
      memcpy(&s->fi[s->nh], s->lbuf, s->nlb * sizeof(uint16_t));
      s->nh += s->nlb;
    }
  }
  /* swap (:497-500) */
#define SWAPP(a, b) do { void* tmp_ = (void*)(a); (a) = (void*)(b); (b) = tmp_; } while (0)
#define SWAPZ(a, b) do { size_t tmp_ = (a); (a) = (b); (b) = tmp_; } while (0)
  { double* t0 = c->v; c->v = s->v; s->v = t0; SWAPZ(c->cap_v, s->cap_v); c->nv = s->nv; }
  { uint8_t* t0 = c->fc; c->fc = s->fc; s->fc = t0; SWAPZ(c->cap_fc, s->cap_fc); c->nf = s->nf; }
  { int32_t* t0 = c->fn; c->fn = s->fn; s->fn = t0; SWAPZ(c->cap_fn, s->cap_fn); }
  { uint16_t* t0 = c->fi; c->fi = s->fi; s->fi = t0; SWAPZ(c->cap_fi, s->cap_fi); c->nh = s->nh; }
#undef SWAPP
#undef SWAPZ
  *r2 = max_d2;
  return 1;
}

/* volume (cell_3d_faces.rs:106-143) and centroid (:145-205).  The two share
 * the per-triangle determinant expression, so one pass yields both with the
 * same bits as two separate passes. */
static void cell_measure(const vdo_cell* c, double* vol, double* cen, uint64_t* cnt) {
  double volume = 0.0, cx = 0.0, cy = 0.0, cz = 0.0, total = 0.0;
  size_t off = 0;
  for (size_t f = 0; f < c->nf; ++f) {
    size_t count = c->fc[f];
    if (count < 3) { off += count; continue; }
    size_t i0 = c->fi[off];
    double v0x = c->v[i0 * 3], v0y = c->v[i0 * 3 + 1], v0z = c->v[i0 * 3 + 2];
    for (size_t i = 1; i < count - 1; ++i) {
      size_t i1 = c->fi[off + i], i2 = c->fi[off + i + 1];
      double v1x = c->v[i1 * 3], v1y = c->v[i1 * 3 + 1], v1z = c->v[i1 * 3 + 2];
      double v2x = c->v[i2 * 3], v2y = c->v[i2 * 3 + 1], v2z = c->v[i2 * 3 + 2];
      volume += v0x * (v1y * v2z - v1z * v2y) + v0y * (v1z * v2x - v1x * v2z) +
                v0z * (v1x * v2y - v1y * v2x);
      double crx = v1y * v2z - v1z * v2y;
      double cry = v1z * v2x - v1x * v2z;
      double crz = v1x * v2y - v1y * v2x;
      double det = v0x * crx + v0y * cry + v0z * crz;
      total += det;
      double tx = v0x + v1x + v2x, ty = v0y + v1y + v2y, tz = v0z + v1z + v2z;
      cx += det * tx; cy += det * ty; cz += det * tz;
      if (cnt) cnt[VDO_CNT_TRIANGLES]++;
    }
    off += count;
  }
  if (vol) *vol = fabs(volume / 6.0);
  if (cen) {
    if (fabs(total) < 1e-9) {
      cen[0] = cen[1] = cen[2] = 0.0;
    } else {
      double factor = 1.0 / (4.0 * total);
      cen[0] = cx * factor; cen[1] = cy * factor; cen[2] = cz * factor;
    }
  }
}

/* face_area (cell_3d_faces.rs:207-254) for a face starting at `off` */
static double face_area_at(const vdo_cell* c, size_t off, size_t count) {
  if (count < 3) return 0.0;
  double area = 0.0;
  size_t p0 = c->fi[off];
  double p0x = c->v[p0 * 3], p0y = c->v[p0 * 3 + 1], p0z = c->v[p0 * 3 + 2];
  for (size_t i = 1; i < count - 1; ++i) {
    size_t p1 = c->fi[off + i], p2 = c->fi[off + i + 1];
    double v1x = c->v[p1 * 3] - p0x, v1y = c->v[p1 * 3 + 1] - p0y, v1z = c->v[p1 * 3 + 2] - p0z;
    double v2x = c->v[p2 * 3] - p0x, v2y = c->v[p2 * 3 + 1] - p0y, v2z = c->v[p2 * 3 + 2] - p0z;
    double crx = v1y * v2z - v1z * v2y;
    double cry = v1z * v2x - v1x * v2z;
    double crz = v1x * v2y - v1y * v2x;
    area += 0.5 * sqrt(crx * crx + cry * cry + crz * crz);
  }
  return area;
}

/* ------------------------------------------------------------------ */
/* walls (wall_3d.rs:8-101, wall/mod.rs)                                */
/* ------------------------------------------------------------------ */
#define VDO_MAX_PLANES 64
typedef struct {
  int kind; /* 0 plane, 1 sphere, 2 cylinder, 3 cone, 4 torus, 5 convex polyhedron */
  int32_t id;
  double a[3]; /* plane point / sphere, cylinder, torus centre / cone tip */
  double n[3]; /* plane normal (points IN) / cylinder, cone, torus axis (normalised) */
  double r;    /* sphere, cylinder radius / torus major radius / cone half-angle */
  double r2;   /* torus minor radius */
  int np;      /* convex polyhedron: planes (point, normal pointing OUT) */
  double planes[VDO_MAX_PLANES][6];
} wall_t;

/* WallGeometry::contains for each kind (wall_3d.rs:31-36, 73-78, 132-143,
 * 202-214, 293-309, 691-701) */
static int wall_contains(const wall_t* w, const double* p) {
  double dx = p[0] - w->a[0], dy = p[1] - w->a[1], dz = p[2] - w->a[2];
  switch (w->kind) {
    case 0: return (dx * w->n[0] + dy * w->n[1] + dz * w->n[2]) >= 0.0;
    case 1: return (dx * dx + dy * dy + dz * dz) <= w->r * w->r;
    case 2: {
      double dot = dx * w->n[0] + dy * w->n[1] + dz * w->n[2];
      double px = dx - dot * w->n[0], py = dy - dot * w->n[1], pz = dz - dot * w->n[2];
      return (px * px + py * py + pz * pz) <= w->r * w->r;
    }
    case 3: {
      double h = dx * w->n[0] + dy * w->n[1] + dz * w->n[2];
      double px = dx - h * w->n[0], py = dy - h * w->n[1], pz = dz - h * w->n[2];
      double r = sqrt(px * px + py * py + pz * pz);
      return h >= 0.0 && r <= h * tan(w->r);
    }
    case 4: {
      double dot = dx * w->n[0] + dy * w->n[1] + dz * w->n[2];
      double px = dx - dot * w->n[0], py = dy - dot * w->n[1], pz = dz - dot * w->n[2];
      double dp = sqrt(px * px + py * py + pz * pz);
      double q = dp - w->r;
      return sqrt(q * q + dot * dot) <= w->r2;
    }
    default:
      for (int k = 0; k < w->np; ++k) {
        const double* pl = w->planes[k];
        double ex = p[0] - pl[0], ey = p[1] - pl[1], ez = p[2] - pl[2];
        if (ex * pl[3] + ey * pl[4] + ez * pl[5] > 0.0) return 0;
      }
      return 1;
  }
}

/* WallGeometry::cut for one generator: the planes (point, outward normal) it
 * emits, in order, into p/n; returns their count */
static int wall_cut(const wall_t* w, const double* g, double* p, double* n) {
  switch (w->kind) {
    case 0: /* wall_3d.rs:38-42 */
      p[0] = w->a[0]; p[1] = w->a[1]; p[2] = w->a[2];
      n[0] = -w->n[0]; n[1] = -w->n[1]; n[2] = -w->n[2];
      return 1;
    case 1: { /* wall_3d.rs:80-100 */
      double dx = g[0] - w->a[0], dy = g[1] - w->a[1], dz = g[2] - w->a[2];
      double dist = sqrt(dx * dx + dy * dy + dz * dz);
      if (dist == 0.0) return 0;
      double scale = w->r / dist;
      p[0] = w->a[0] + dx * scale; p[1] = w->a[1] + dy * scale; p[2] = w->a[2] + dz * scale;
      n[0] = dx / dist; n[1] = dy / dist; n[2] = dz / dist;
      return 1;
    }
    case 2: { /* wall_3d.rs:145-173 */
      double dx = g[0] - w->a[0], dy = g[1] - w->a[1], dz = g[2] - w->a[2];
      double dot = dx * w->n[0] + dy * w->n[1] + dz * w->n[2];
      double px = dx - dot * w->n[0], py = dy - dot * w->n[1], pz = dz - dot * w->n[2];
      double dist = sqrt(px * px + py * py + pz * pz);
      if (dist == 0.0) return 0;
      double scale = w->r / dist;
      p[0] = w->a[0] + dot * w->n[0] + px * scale;
      p[1] = w->a[1] + dot * w->n[1] + py * scale;
      p[2] = w->a[2] + dot * w->n[2] + pz * scale;
      n[0] = px / dist; n[1] = py / dist; n[2] = pz / dist;
      return 1;
    }
    case 3: { /* wall_3d.rs:216-261 */
      double dx = g[0] - w->a[0], dy = g[1] - w->a[1], dz = g[2] - w->a[2];
      double h = dx * w->n[0] + dy * w->n[1] + dz * w->n[2];
      double px = dx - h * w->n[0], py = dy - h * w->n[1], pz = dz - h * w->n[2];
      double r = sqrt(px * px + py * py + pz * pz);
      if (r == 0.0) return 0;
      double rdx = px / r, rdy = py / r, rdz = pz / r;
      double ca = cos(w->r), sa = sin(w->r);
      double dist = r * ca - h * sa;
      double pr = r - dist * ca;
      double ph = h + dist * sa;
      if (ph < 0.0) {
        double dt = sqrt(dx * dx + dy * dy + dz * dz);
        if (dt == 0.0) return 0;
        p[0] = w->a[0]; p[1] = w->a[1]; p[2] = w->a[2];
        n[0] = dx / dt; n[1] = dy / dt; n[2] = dz / dt;
        return 1;
      }
      p[0] = w->a[0] + ph * w->n[0] + pr * rdx;
      p[1] = w->a[1] + ph * w->n[1] + pr * rdy;
      p[2] = w->a[2] + ph * w->n[2] + pr * rdz;
      n[0] = ca * rdx - sa * w->n[0];
      n[1] = ca * rdy - sa * w->n[1];
      n[2] = ca * rdz - sa * w->n[2];
      return 1;
    }
    case 4: { /* wall_3d.rs:311-364 */
      double dx = g[0] - w->a[0], dy = g[1] - w->a[1], dz = g[2] - w->a[2];
      double dot = dx * w->n[0] + dy * w->n[1] + dz * w->n[2];
      double px = dx - dot * w->n[0], py = dy - dot * w->n[1], pz = dz - dot * w->n[2];
      double dp = sqrt(px * px + py * py + pz * pz);
      double ux, uy, uz;
      if (dp < 1e-9) {
        double tx = 1.0, ty = 0.0, tz = 0.0;
        if (fabs(w->n[0]) > 0.9) { tx = 0.0; ty = 1.0; }
        double td = tx * w->n[0] + ty * w->n[1] + tz * w->n[2];
        double ax = tx - td * w->n[0], ay = ty - td * w->n[1], az = tz - td * w->n[2];
        double len = sqrt(ax * ax + ay * ay + az * az);
        if (len == 0.0) return 0;
        ux = ax / len; uy = ay / len; uz = az / len;
      } else {
        ux = px / dp; uy = py / dp; uz = pz / dp;
      }
      double cx = w->a[0] + ux * w->r, cy = w->a[1] + uy * w->r, cz = w->a[2] + uz * w->r;
      double vx = g[0] - cx, vy = g[1] - cy, vz = g[2] - cz;
      double dc = sqrt(vx * vx + vy * vy + vz * vz);
      if (dc == 0.0) return 0;
      n[0] = vx / dc; n[1] = vy / dc; n[2] = vz / dc;
      p[0] = cx + n[0] * w->r2; p[1] = cy + n[1] * w->r2; p[2] = cz + n[2] * w->r2;
      return 1;
    }
    default: /* wall_3d.rs:703-707 */
      for (int k = 0; k < w->np; ++k) {
        memcpy(&p[3 * k], &w->planes[k][0], 3 * sizeof(double));
        memcpy(&n[3 * k], &w->planes[k][3], 3 * sizeof(double));
      }
      return w->np;
  }
}

/* ------------------------------------------------------------------ */
/* tessellation + grid                                                  */
/* ------------------------------------------------------------------ */
typedef struct {
  int32_t dx, dy, dz;
  long long lin; /* enumeration index: ties keep this order */
  double min_d2;
} offset_t;

struct vdo_tess {
  double bmin[3], bmax[3];
  size_t nx, ny, nz;
  double sx, sy, sz;       /* grid_scale */
  double lx, ly, lz;       /* grid_limit = n - 1e-5 */
  offset_t* order; size_t norder;
  /* a truncated order (vdo_create_truncated) holds every entry with
   * min_d2 < order_bound; cells whose walk reaches its end unfinished are
   * counted in `exhausted` */
  int truncated; double order_bound; size_t exhausted;
  wall_t walls[VDO_MAX_WALLS]; int nwalls;
  double* gen; size_t ngen;
  size_t* bin_of;          /* generator_bin_ids */
  size_t* bin_start;       /* CSR of grid_bins, members in the reference's push order */
  size_t* bin_members;
  vdo_cell* cells; size_t ncells;
  uint64_t counters[VDO_NCOUNTERS];
  /* seal_log, prune_log, prune_pos_log (tessellation.rs:19-21) */
  int32_t* seal_log; size_t nseal, cap_seal;
  int32_t* prune_log; size_t nprune, cap_prune;
  double* prune_pos; size_t nprune_pos, cap_prune_pos;
};

static int cmp_offset(const void* a, const void* b) {
  const offset_t* x = (const offset_t*)a;
  const offset_t* y = (const offset_t*)b;
  if (x->min_d2 < y->min_d2) return -1;
  if (x->min_d2 > y->min_d2) return 1;
  return (x->lin > y->lin) - (x->lin < y->lin);
}

/* Algorithm3DGrid::new (algo_3d_grid.rs:47-95), stable tie order.
 * k > 0 keeps only the offsets with |dx|, |dy|, |dz| <= k, each with its
 * enumeration index in the complete table, so the kept entries are in the
 * complete table's order; every omitted entry has min_d2 >= the smallest
 * (k cs)^2 over the truncated axes, and a walk that breaks before reaching
 * that bound visits exactly what the complete table gives it. */
vdo_tess* vdo_create_truncated(const double bmin[3], const double bmax[3], int nx, int ny, int nz, int k) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return NULL;
  vdo_tess* t = (vdo_tess*)calloc(1, sizeof(vdo_tess));
  memcpy(t->bmin, bmin, 3 * sizeof(double));
  memcpy(t->bmax, bmax, 3 * sizeof(double));
  t->nx = (size_t)nx; t->ny = (size_t)ny; t->nz = (size_t)nz;
  t->sx = (double)nx / (bmax[0] - bmin[0]);
  t->sy = (double)ny / (bmax[1] - bmin[1]);
  t->sz = (double)nz / (bmax[2] - bmin[2]);
  t->lx = (double)nx - 1e-5; t->ly = (double)ny - 1e-5; t->lz = (double)nz - 1e-5;
  double csx = 1.0 / t->sx, csy = 1.0 / t->sy, csz = 1.0 / t->sz;
  const int kx = (k > 0 && k < nx) ? k : nx, ky = (k > 0 && k < ny) ? k : ny, kz = (k > 0 && k < nz) ? k : nz;
  t->truncated = kx < nx || ky < ny || kz < nz;
  t->order_bound = INFINITY;
  if (kx < nx) t->order_bound = fmin(t->order_bound, ((double)kx * csx) * ((double)kx * csx));
  if (ky < ny) t->order_bound = fmin(t->order_bound, ((double)ky * csy) * ((double)ky * csy));
  if (kz < nz) t->order_bound = fmin(t->order_bound, ((double)kz * csz) * ((double)kz * csz));
  size_t n = (size_t)(2 * kx + 1) * (size_t)(2 * ky + 1) * (size_t)(2 * kz + 1);
  t->order = (offset_t*)malloc(n * sizeof(offset_t));
  size_t q = 0;
  for (int z = -kz; z <= kz; ++z)
    for (int y = -ky; y <= ky; ++y)
      for (int x = -kx; x <= kx; ++x) {
        double mx = x > 0 ? (double)(x - 1) * csx : (x < 0 ? (double)(-x - 1) * csx : 0.0);
        double my = y > 0 ? (double)(y - 1) * csy : (y < 0 ? (double)(-y - 1) * csy : 0.0);
        double mz = z > 0 ? (double)(z - 1) * csz : (z < 0 ? (double)(-z - 1) * csz : 0.0);
        /* the index in the complete z-outer, x-inner enumeration */
        long long lin = (((long long)z + nz) * (2LL * ny + 1) + ((long long)y + ny)) * (2LL * nx + 1) + (x + nx);
        offset_t o = {x, y, z, lin, mx * mx + my * my + mz * mz};
        t->order[q++] = o;
      }
  qsort(t->order, n, sizeof(offset_t), cmp_offset);
  t->norder = n;
  t->bin_start = (size_t*)calloc(t->nx * t->ny * t->nz + 1, sizeof(size_t));
  return t;
}

vdo_tess* vdo_create(const double bmin[3], const double bmax[3], int nx, int ny, int nz) {
  return vdo_create_truncated(bmin, bmax, nx, ny, nz, 0);
}

size_t vdo_table_exhausted(const vdo_tess* t) { return t->exhausted; }

static void free_cells(vdo_tess* t) {
  for (size_t i = 0; i < t->ncells; ++i) {
    free(t->cells[i].v); free(t->cells[i].fc); free(t->cells[i].fn); free(t->cells[i].fi);
  }
  free(t->cells);
  t->cells = NULL;
  t->ncells = 0;
}

void vdo_destroy(vdo_tess* t) {
  if (!t) return;
  free_cells(t);
  free(t->order); free(t->gen); free(t->bin_of); free(t->bin_start); free(t->bin_members);
  free(t->seal_log); free(t->prune_log); free(t->prune_pos);
  free(t);
}

static inline size_t to_index(double v) {
  /* `f64 as usize`: saturating, NaN -> 0 */
  if (!(v > 0.0)) return 0;
  return (size_t)v;
}
static inline double clampd(double v, double lo, double hi) {
  if (v < lo) return lo;
  if (v > hi) return hi;
  return v;
}

/* get_bin_index (algo_3d_grid.rs:98-107) */
size_t vdo_bin_index(const vdo_tess* t, double x, double y, double z) {
  size_t ix = to_index(clampd((x - t->bmin[0]) * t->sx, 0.0, t->lx));
  size_t iy = to_index(clampd((y - t->bmin[1]) * t->sy, 0.0, t->ly));
  size_t iz = to_index(clampd((z - t->bmin[2]) * t->sz, 0.0, t->lz));
  return ix + iy * t->nx + iz * t->nx * t->ny;
}

/* Algorithm3DGrid::set_generators (algo_3d_grid.rs:111-130) */
static void grid_rebin(vdo_tess* t) {
  size_t nb = t->nx * t->ny * t->nz;
  free(t->bin_of); free(t->bin_members);
  t->bin_of = (size_t*)malloc((t->ngen ? t->ngen : 1) * sizeof(size_t));
  t->bin_members = (size_t*)malloc((t->ngen ? t->ngen : 1) * sizeof(size_t));
  memset(t->bin_start, 0, (nb + 1) * sizeof(size_t));
  for (size_t i = 0; i < t->ngen; ++i) {
    size_t b = vdo_bin_index(t, t->gen[3 * i], t->gen[3 * i + 1], t->gen[3 * i + 2]);
    t->bin_of[i] = b;
    t->bin_start[b + 1]++;
  }
  for (size_t b = 0; b < nb; ++b) t->bin_start[b + 1] += t->bin_start[b];
  size_t* cur = (size_t*)malloc((nb ? nb : 1) * sizeof(size_t));
  memcpy(cur, t->bin_start, nb * sizeof(size_t));
  for (size_t i = 0; i < t->ngen; ++i) t->bin_members[cur[t->bin_of[i]]++] = i;
  free(cur);
}

static int walls_contain(const vdo_tess* t, const double* p) {
  for (int w = 0; w < t->nwalls; ++w)
    if (!wall_contains(&t->walls[w], p)) return 0;
  return 1;
}

/* Tessellation::set_generators (tessellation.rs:43-67): walls only */
size_t vdo_set_generators(vdo_tess* t, const double* xyz, size_t n) {
  double* keep = (double*)malloc((n ? n : 1) * 3 * sizeof(double));
  size_t m = 0;
  for (size_t i = 0; i < n; ++i) {
    if (walls_contain(t, &xyz[3 * i])) {
      memcpy(&keep[3 * m], &xyz[3 * i], 3 * sizeof(double));
      m++;
    }
  }
  free(t->gen);
  t->gen = keep;
  t->ngen = m;
  grid_rebin(t);
  return m;
}

/* Tessellation::set_generator (tessellation.rs:70-92) and
   Algorithm3DGrid::update_generator (algo_3d_grid.rs:132-143): ignored when the
   index is out of range or a wall does not contain the point; a bin change
   swap_removes the id from its old bin and pushes it onto the new one, so the
   in-bin visit order is the reference's. */
void vdo_set_generator(vdo_tess* t, size_t index, const double xyz[3]) {
  if (index >= t->ngen || !walls_contain(t, xyz)) return;
  const size_t nb = t->nx * t->ny * t->nz;
  const size_t nbin = vdo_bin_index(t, xyz[0], xyz[1], xyz[2]), ob = t->bin_of[index];
  if (nbin != ob) {
    size_t pos = t->bin_start[ob];
    while (t->bin_members[pos] != index) ++pos;
    const size_t last = t->bin_start[ob + 1] - 1;
    t->bin_members[pos] = t->bin_members[last];
    size_t* mem = (size_t*)malloc(t->ngen * sizeof(size_t));
    size_t m = 0;
    for (size_t b = 0; b < nb; ++b) {
      const size_t s = t->bin_start[b], e = b == ob ? last : t->bin_start[b + 1];
      t->bin_start[b] = m;
      for (size_t k = s; k < e; ++k) mem[m++] = t->bin_members[k];
      if (b == nbin) mem[m++] = index;
    }
    t->bin_start[nb] = m;
    free(t->bin_members);
    t->bin_members = mem;
    t->bin_of[index] = nbin;
  }
  memcpy(&t->gen[3 * index], xyz, 3 * sizeof(double));
}

/* SplitMix64 (Steele, Lea & Flood, OOPSLA 2014) as a counter-based generator:
   draw k of a seed mixes seed + (k + 1) * 0x9e3779b97f4a7c15. */
static uint64_t splitmix64_at(uint64_t seed, uint64_t k) {
  uint64_t z = seed + (k + 1) * 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

/* Tessellation::random_generators (tessellation.rs:96-121) with an explicit
   seed in place of thread_rng: attempts one at a time, each coordinate
   min + u * (max - min) with u = (draw >> 11) * 2^-53, kept when every wall
   contains the point, until `count` are kept or count * 1000 attempts. */
size_t vdo_random_generators(vdo_tess* t, size_t count, uint64_t seed) {
  double* pts = (double*)malloc((count ? count : 1) * 3 * sizeof(double));
  size_t found = 0;
  const uint64_t max_attempts = (uint64_t)count * 1000u;
  for (uint64_t a = 0; found < count && a < max_attempts; ++a) {
    double p[3];
    for (int c = 0; c < 3; ++c) {
      const double u = (double)(splitmix64_at(seed, 3 * a + (uint64_t)c) >> 11) * 0x1p-53;
      p[c] = t->bmin[c] + u * (t->bmax[c] - t->bmin[c]);
    }
    if (walls_contain(t, p)) {
      memcpy(&pts[3 * found], p, sizeof(p));
      found++;
    }
  }
  free(t->gen);
  t->gen = pts;
  t->ngen = found;
  grid_rebin(t);
  return found;
}

/* prune_outside_generators + add_wall (tessellation.rs:175-200) */
static int add_wall(vdo_tess* t, const wall_t* w) {
  if (w->id > VDO_WALL_ID_MAX || t->nwalls >= VDO_MAX_WALLS) return -1;
  t->walls[t->nwalls++] = *w;
  size_t m = 0;
  for (size_t i = 0; i < t->ngen; ++i) {
    if (walls_contain(t, &t->gen[3 * i])) {
      if (m != i) memmove(&t->gen[3 * m], &t->gen[3 * i], 3 * sizeof(double));
      m++;
    }
  }
  if (m != t->ngen) {
    t->ngen = m;
    grid_rebin(t);
  }
  return 0;
}

int vdo_add_wall_plane(vdo_tess* t, const double point[3], const double normal[3], int id) {
  wall_t w;
  memset(&w, 0, sizeof(w));
  w.kind = 0; w.id = id;
  memcpy(w.a, point, 3 * sizeof(double));
  /* PlaneGeometry::new (wall_3d.rs:23-27) */
  double len = sqrt(normal[0] * normal[0] + normal[1] * normal[1] + normal[2] * normal[2]);
  if (len == 0.0) { w.n[0] = 0.0; w.n[1] = 0.0; w.n[2] = 1.0; }
  else { w.n[0] = normal[0] / len; w.n[1] = normal[1] / len; w.n[2] = normal[2] / len; }
  return add_wall(t, &w);
}

int vdo_add_wall_sphere(vdo_tess* t, const double center[3], double radius, int id) {
  wall_t w;
  memset(&w, 0, sizeof(w));
  w.kind = 1; w.id = id; w.r = radius;
  memcpy(w.a, center, 3 * sizeof(double));
  return add_wall(t, &w);
}

/* an axis normalised as in CylinderGeometry/ConeGeometry/TorusGeometry::new
 * (wall_3d.rs:124-128, 194-198, 285-289) */
static void unit_axis(const double axis[3], double out[3]) {
  double len = sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
  if (len == 0.0) { out[0] = 0.0; out[1] = 0.0; out[2] = 1.0; }
  else { out[0] = axis[0] / len; out[1] = axis[1] / len; out[2] = axis[2] / len; }
}

int vdo_add_wall_cylinder(vdo_tess* t, const double center[3], const double axis[3], double radius, int id) {
  wall_t w;
  memset(&w, 0, sizeof(w));
  w.kind = 2; w.id = id; w.r = radius;
  memcpy(w.a, center, 3 * sizeof(double));
  unit_axis(axis, w.n);
  return add_wall(t, &w);
}

int vdo_add_wall_cone(vdo_tess* t, const double tip[3], const double axis[3], double angle, int id) {
  wall_t w;
  memset(&w, 0, sizeof(w));
  w.kind = 3; w.id = id; w.r = angle;
  memcpy(w.a, tip, 3 * sizeof(double));
  unit_axis(axis, w.n);
  return add_wall(t, &w);
}

int vdo_add_wall_torus(vdo_tess* t, const double center[3], const double axis[3], double major, double minor,
                       int id) {
  wall_t w;
  memset(&w, 0, sizeof(w));
  w.kind = 4; w.id = id; w.r = major; w.r2 = minor;
  memcpy(w.a, center, 3 * sizeof(double));
  unit_axis(axis, w.n);
  return add_wall(t, &w);
}

/* ConvexPolyhedronGeometry::new (wall_3d.rs:476-492): planes (point, normal
 * pointing OUT), taken as given */
int vdo_add_wall_polyhedron(vdo_tess* t, const double* points, const double* normals, int nplanes, int id) {
  if (nplanes < 0 || nplanes > VDO_MAX_PLANES) return -1;
  wall_t w;
  memset(&w, 0, sizeof(w));
  w.kind = 5; w.id = id; w.np = nplanes;
  for (int k = 0; k < nplanes; ++k) {
    memcpy(&w.planes[k][0], &points[3 * k], 3 * sizeof(double));
    memcpy(&w.planes[k][3], &normals[3 * k], 3 * sizeof(double));
  }
  return add_wall(t, &w);
}

/* the regular polyhedra of ConvexPolyhedronGeometry::new_* (wall_3d.rs:499-688):
 * kind 4 tetrahedron, 6 hexahedron, 8 octahedron, 12 dodecahedron,
 * 20 icosahedron; returns the plane count or -1 */
int vdo_regular_polyhedron(int kind, const double center[3], double radius, double* points, double* normals) {
  double bn[20][3];
  int m = 0, unit = 1;
  double dist;
  if (kind == 4) {
    static const double b[4][3] = {{-1, -1, -1}, {-1, 1, 1}, {1, -1, 1}, {1, 1, -1}};
    memcpy(bn, b, sizeof(b)); m = 4;
    dist = radius / 3.0;
  } else if (kind == 6) {
    static const double b[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    memcpy(bn, b, sizeof(b)); m = 6; unit = 0; /* used as given, not normalised */
    dist = radius / sqrt(3.0);
  } else if (kind == 8) {
    for (int x = -1; x <= 1; x += 2)
      for (int y = -1; y <= 1; y += 2)
        for (int z = -1; z <= 1; z += 2) { bn[m][0] = x; bn[m][1] = y; bn[m][2] = z; ++m; }
    dist = radius / sqrt(3.0);
  } else if (kind == 12) {
    double phi = (1.0 + sqrt(5.0)) / 2.0;
    double xi = sqrt((5.0 + 2.0 * sqrt(5.0)) / 15.0);
    dist = radius * xi;
    const double b[12][3] = {{0.0, phi, 1.0}, {0.0, -phi, 1.0}, {0.0, phi, -1.0}, {0.0, -phi, -1.0},
                             {1.0, 0.0, phi}, {1.0, 0.0, -phi}, {-1.0, 0.0, phi}, {-1.0, 0.0, -phi},
                             {phi, 1.0, 0.0}, {phi, -1.0, 0.0}, {-phi, 1.0, 0.0}, {-phi, -1.0, 0.0}};
    memcpy(bn, b, sizeof(b)); m = 12;
  } else if (kind == 20) {
    double phi = (1.0 + sqrt(5.0)) / 2.0;
    double xi = sqrt((5.0 + 2.0 * sqrt(5.0)) / 15.0);
    dist = radius * xi;
    double ip = 1.0 / phi;
    for (int x = -1; x <= 1; x += 2)
      for (int y = -1; y <= 1; y += 2)
        for (int z = -1; z <= 1; z += 2) { bn[m][0] = x; bn[m][1] = y; bn[m][2] = z; ++m; }
    for (int y = -1; y <= 1; y += 2)
      for (int z = -1; z <= 1; z += 2) { bn[m][0] = 0.0; bn[m][1] = y * phi; bn[m][2] = z * ip; ++m; }
    for (int x = -1; x <= 1; x += 2)
      for (int z = -1; z <= 1; z += 2) { bn[m][0] = x * ip; bn[m][1] = 0.0; bn[m][2] = z * phi; ++m; }
    for (int x = -1; x <= 1; x += 2)
      for (int y = -1; y <= 1; y += 2) { bn[m][0] = x * phi; bn[m][1] = y * ip; bn[m][2] = 0.0; ++m; }
  } else {
    return -1;
  }
  for (int k = 0; k < m; ++k) {
    double nx = bn[k][0], ny = bn[k][1], nz = bn[k][2];
    if (unit) {
      double len = sqrt(nx * nx + ny * ny + nz * nz);
      nx = nx / len; ny = ny / len; nz = nz / len;
    }
    normals[3 * k] = nx; normals[3 * k + 1] = ny; normals[3 * k + 2] = nz;
    points[3 * k] = center[0] + nx * dist;
    points[3 * k + 1] = center[1] + ny * dist;
    points[3 * k + 2] = center[2] + nz * dist;
  }
  return m;
}

void vdo_clear_walls(vdo_tess* t) { t->nwalls = 0; }

/* compute_cell (tessellation.rs:414-475) with visit_neighbors
 * (algo_3d_grid.rs:145-202) and the visitor (tessellation.rs:446-471) */
/* returns 1 when the walk ran off a truncated search order unfinished */
static int compute_cell(const vdo_tess* t, size_t i, vdo_cell* cell, scratch_t* s, uint64_t* cnt) {
  const double g[3] = {t->gen[3 * i], t->gen[3 * i + 1], t->gen[3 * i + 2]};
  double r2;
  cell_init_box(cell, i, t->bmin, t->bmax);
  for (int w = 0; w < t->nwalls; ++w) {
    double p[3 * VDO_MAX_PLANES], n[3 * VDO_MAX_PLANES];
    int np = wall_cut(&t->walls[w], g, p, n);
    for (int k = 0; k < np; ++k) cell_clip(cell, &p[3 * k], &n[3 * k], t->walls[w].id, s, NULL, &r2, cnt);
    if (cell->nv == 0) return 0;
  }
  double cur = cell_max_radius_sq(cell, g);

  size_t b = t->bin_of[i];
  size_t nxy = t->nx * t->ny;
  size_t iz = b / nxy, rem = b % nxy, iy = rem / t->nx, ix = rem % t->nx;
  double csx = 1.0 / t->sx, csy = 1.0 / t->sy, csz = 1.0 / t->sz;
  double rx = (g[0] - t->bmin[0]) * t->sx - (double)ix;
  double ry = (g[1] - t->bmin[1]) * t->sy - (double)iy;
  double rz = (g[2] - t->bmin[2]) * t->sz - (double)iz;
  int broke = 0;
  for (size_t k = 0; k < t->norder; ++k) {
    const offset_t* o = &t->order[k];
    if (cnt) cnt[VDO_CNT_OFFSETS]++;
    if (o->min_d2 > 4.0 * cur) {
      broke = 1;
      break;
    }
    long bx = (long)ix + o->dx, by = (long)iy + o->dy, bz = (long)iz + o->dz;
    if (bx < 0 || bx >= (long)t->nx || by < 0 || by >= (long)t->ny || bz < 0 || bz >= (long)t->nz)
      continue;
    double ddx = o->dx > 0 ? ((double)o->dx - rx) * csx : (o->dx < 0 ? ((double)(-(o->dx + 1)) + rx) * csx : 0.0);
    double ddy = o->dy > 0 ? ((double)o->dy - ry) * csy : (o->dy < 0 ? ((double)(-(o->dy + 1)) + ry) * csy : 0.0);
    double ddz = o->dz > 0 ? ((double)o->dz - rz) * csz : (o->dz < 0 ? ((double)(-(o->dz + 1)) + rz) * csz : 0.0);
    double bdx = fmax(ddx, 0.0), bdy = fmax(ddy, 0.0), bdz = fmax(ddz, 0.0);
    if (!(bdx * bdx + bdy * bdy + bdz * bdz <= 4.0 * cur)) continue;
    size_t bin = (size_t)bx + (size_t)by * t->nx + (size_t)bz * nxy;
    for (size_t m = t->bin_start[bin]; m < t->bin_start[bin + 1]; ++m) {
      size_t j = t->bin_members[m];
      if (j == i) continue;
      if (cnt) cnt[VDO_CNT_CANDIDATES]++;
      const double* q = &t->gen[3 * j];
      double dist_sq = 0.0, mid[3], nrm[3];
      for (int a = 0; a < 3; ++a) {
        double d = q[a] - g[a];
        dist_sq += d * d;
        mid[a] = g[a] + d * 0.5;
        nrm[a] = d;
      }
      if (dist_sq > 4.0 * cur) continue;
      if (cell_clip(cell, mid, nrm, (int32_t)j, s, g, &r2, cnt)) {
        cur = (cell->nv == 0) ? 0.0 : r2;
      }
    }
  }
  return t->truncated && !broke && !(t->order_bound > 4.0 * cur);
}

void vdo_calculate_range(vdo_tess* t, size_t begin, size_t end, int nthreads) {
  /* calculate clears the logs (tessellation.rs:214-216) */
  t->nseal = 0; t->nprune = 0; t->nprune_pos = 0;
  free_cells(t);
  t->ncells = t->ngen;
  t->cells = (vdo_cell*)calloc(t->ncells ? t->ncells : 1, sizeof(vdo_cell));
  memset(t->counters, 0, sizeof(t->counters));
  t->exhausted = 0;
  if (end > t->ngen) end = t->ngen;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
  {
    scratch_t s;
    memset(&s, 0, sizeof(s));
    uint64_t cnt[VDO_NCOUNTERS];
    memset(cnt, 0, sizeof(cnt));
    size_t exh = 0;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
    for (long long i = (long long)begin; i < (long long)end; ++i) {
      exh += (size_t)compute_cell(t, (size_t)i, &t->cells[i], &s, cnt);
      cell_measure(&t->cells[i], NULL, NULL, cnt);
    }
#ifdef _OPENMP
#pragma omp critical
#endif
    {
      for (int k = 0; k < VDO_NCOUNTERS; ++k) t->counters[k] += cnt[k];
      t->exhausted += exh;
    }
    scratch_free(&s);
  }
  (void)nthreads;
}

void vdo_calculate(vdo_tess* t, int nthreads) { vdo_calculate_range(t, 0, t->ngen, nthreads); }

/* ------------------------------------------------------------------ */
/* calculate_sealed / prune_boundaries (tessellation.rs:234-385)        */
/* ------------------------------------------------------------------ */
/* WallGeometry::is_planar: planes and convex polyhedra (wall_3d.rs:44-46, 710-712) */
static int wall_planar(const wall_t* w) { return w->kind == 0 || w->kind == 5; }

static int has_id(const int32_t* a, size_t n, int32_t x) {
  for (size_t k = 0; k < n; ++k)
    if (a[k] == x) return 1;
  return 0;
}

/* a cell's neighbours (face neighbours in [0, count), face order; distinct
 * only when `dedup`) and its curved walls: distinct face neighbour ids whose
 * first wall with that id (walls.iter().find) is not planar
 * (tessellation.rs:242-261, 333-353) */
static void cell_topology(const vdo_tess* t, const vdo_cell* c, size_t count, int dedup, int32_t* nb,
                          size_t* nnb, int32_t* cw, size_t* ncw) {
  *nnb = 0;
  *ncw = 0;
  for (size_t f = 0; f < c->nf; ++f) {
    int32_t x = c->fn[f];
    if (x >= 0 && (size_t)x < count) {
      if (!dedup || !has_id(nb, *nnb, x)) nb[(*nnb)++] = x;
    } else {
      for (int w = 0; w < t->nwalls; ++w) {
        if (t->walls[w].id != x) continue;
        if (!wall_planar(&t->walls[w]) && !has_id(cw, *ncw, x)) cw[(*ncw)++] = x;
        break;
      }
    }
  }
}

static void log_push_i(int32_t** a, size_t* n, size_t* cap, int32_t x) {
  if (*n == *cap) {
    *cap = *cap ? 2 * *cap : 64;
    *a = (int32_t*)realloc(*a, *cap * sizeof(int32_t));
  }
  (*a)[(*n)++] = x;
}

static void log_push_d(double** a, size_t* n, size_t* cap, double x) {
  if (*n == *cap) {
    *cap = *cap ? 2 * *cap : 64;
    *a = (double*)realloc(*a, *cap * sizeof(double));
  }
  (*a)[(*n)++] = x;
}

typedef struct {
  int32_t* nb; size_t* nnb;  /* per cell, at most nf entries from offset[i] */
  int32_t* cw; size_t* ncw;
  size_t* off;
} topo_t;

static void topo_build(const vdo_tess* t, int dedup, topo_t* T) {
  size_t count = t->ngen, tot = 0;
  T->off = (size_t*)malloc((count + 1) * sizeof(size_t));
  for (size_t i = 0; i < count; ++i) { T->off[i] = tot; tot += t->cells[i].nf; }
  T->off[count] = tot;
  T->nb = (int32_t*)malloc((tot ? tot : 1) * sizeof(int32_t));
  T->cw = (int32_t*)malloc((tot ? tot : 1) * sizeof(int32_t));
  T->nnb = (size_t*)malloc((count ? count : 1) * sizeof(size_t));
  T->ncw = (size_t*)malloc((count ? count : 1) * sizeof(size_t));
  for (size_t i = 0; i < count; ++i)
    cell_topology(t, &t->cells[i], count, dedup, T->nb + T->off[i], &T->nnb[i], T->cw + T->off[i], &T->ncw[i]);
}

static void topo_free(topo_t* T) { free(T->nb); free(T->cw); free(T->nnb); free(T->ncw); free(T->off); }

/* Tessellation::calculate_sealed (tessellation.rs:234-318): calculate, then
 * clip every cell on a curved wall with the wall's tangent plane at each
 * neighbour on the same wall, when its own generator lies on the plane's
 * valid side; the topology is taken before any cell changes */
void vdo_calculate_sealed(vdo_tess* t, int nthreads) {
  vdo_calculate(t, nthreads);
  size_t count = t->ngen;
  topo_t T;
  topo_build(t, 0, &T);
  scratch_t s;
  memset(&s, 0, sizeof(s));
  for (size_t i = 0; i < count; ++i) {
    if (T.ncw[i] == 0) continue;
    const double* g = &t->gen[3 * i];
    const int32_t* nb = T.nb + T.off[i];
    for (size_t q = 0; q < T.nnb[i]; ++q) {
      size_t j = (size_t)nb[q];
      for (int w = 0; w < t->nwalls; ++w) {
        const wall_t* W = &t->walls[w];
        if (wall_planar(W) || !has_id(T.cw + T.off[i], T.ncw[i], W->id) || !has_id(T.cw + T.off[j], T.ncw[j], W->id))
          continue;
        double p[3 * VDO_MAX_PLANES], n[3 * VDO_MAX_PLANES];
        int np = wall_cut(W, &t->gen[3 * j], p, n);
        for (int k = 0; k < np; ++k) {
          double dot = 0.0;
          for (int d = 0; d < 3; ++d) dot += (g[d] - p[3 * k + d]) * n[3 * k + d];
          if (dot <= 1e-9) {
            double r2;
            if (cell_clip(&t->cells[i], &p[3 * k], &n[3 * k], W->id, &s, NULL, &r2, NULL)) {
              log_push_i(&t->seal_log, &t->nseal, &t->cap_seal, (int32_t)i);
              log_push_i(&t->seal_log, &t->nseal, &t->cap_seal, (int32_t)j);
              log_push_i(&t->seal_log, &t->nseal, &t->cap_seal, W->id);
            }
          }
        }
      }
    }
  }
  scratch_free(&s);
  topo_free(&T);
}

/* Cell::shared_vertices (cell_3d_faces.rs:536-565) */
static size_t shared_vertices(const vdo_cell* c, int32_t a, int32_t b, double* out) {
  size_t* av = (size_t*)malloc((c->nh ? c->nh : 1) * sizeof(size_t));
  size_t* bv = (size_t*)malloc((c->nh ? c->nh : 1) * sizeof(size_t));
  size_t na = 0, nbv = 0, off = 0, m = 0;
  for (size_t f = 0; f < c->nf; ++f) {
    size_t cnt = c->fc[f];
    for (size_t k = 0; k < cnt; ++k) {
      size_t v = c->fi[off + k];
      if (c->fn[f] == a) {
        size_t z = 0;
        while (z < na && av[z] != v) ++z;
        if (z == na) av[na++] = v;
      }
      if (c->fn[f] == b) {
        size_t z = 0;
        while (z < nbv && bv[z] != v) ++z;
        if (z == nbv) bv[nbv++] = v;
      }
    }
    off += cnt;
  }
  for (size_t x = 0; x < na; ++x) {
    size_t z = 0;
    while (z < nbv && bv[z] != av[x]) ++z;
    if (z < nbv) {
      memcpy(&out[3 * m], &c->v[3 * av[x]], 3 * sizeof(double));
      ++m;
    }
  }
  free(av);
  free(bv);
  return m;
}

/* Tessellation::prune_boundaries (tessellation.rs:323-385): for every cell
 * on a curved wall and every distinct neighbour on the same wall, the
 * vertices the cell's wall face shares with its face towards the neighbour */
void vdo_prune_boundaries(vdo_tess* t) {
  size_t count = t->ngen;
  t->nprune = 0;
  t->nprune_pos = 0;
  topo_t T;
  topo_build(t, 1, &T);
  for (size_t i = 0; i < count; ++i) {
    if (T.ncw[i] == 0) continue;
    const vdo_cell* c = &t->cells[i];
    double* sh = (double*)malloc((3 * c->nh + 3) * sizeof(double));
    const int32_t* nb = T.nb + T.off[i];
    for (size_t q = 0; q < T.nnb[i]; ++q) {
      size_t j = (size_t)nb[q];
      for (int w = 0; w < t->nwalls; ++w) {
        const wall_t* W = &t->walls[w];
        if (wall_planar(W) || !has_id(T.cw + T.off[i], T.ncw[i], W->id) || !has_id(T.cw + T.off[j], T.ncw[j], W->id))
          continue;
        size_t m = shared_vertices(c, W->id, (int32_t)j, sh);
        if (m == 0) continue;
        log_push_i(&t->prune_log, &t->nprune, &t->cap_prune, (int32_t)i);
        log_push_i(&t->prune_log, &t->nprune, &t->cap_prune, (int32_t)j);
        log_push_i(&t->prune_log, &t->nprune, &t->cap_prune, W->id);
        log_push_i(&t->prune_log, &t->nprune, &t->cap_prune, (int32_t)m);
        for (size_t k = 0; k < 3 * m; ++k) log_push_d(&t->prune_pos, &t->nprune_pos, &t->cap_prune_pos, sh[k]);
      }
    }
    free(sh);
  }
  topo_free(&T);
}

size_t vdo_seal_log_len(const vdo_tess* t) { return t->nseal; }
void vdo_get_seal_log(const vdo_tess* t, int32_t* out) { if (t->nseal) memcpy(out, t->seal_log, t->nseal * sizeof(int32_t)); }
size_t vdo_prune_log_len(const vdo_tess* t) { return t->nprune; }
void vdo_get_prune_log(const vdo_tess* t, int32_t* out) { if (t->nprune) memcpy(out, t->prune_log, t->nprune * sizeof(int32_t)); }
size_t vdo_prune_pos_log_len(const vdo_tess* t) { return t->nprune_pos; }
void vdo_get_prune_pos_log(const vdo_tess* t, double* out) {
  if (t->nprune_pos) memcpy(out, t->prune_pos, t->nprune_pos * sizeof(double));
}

/* Tessellation::relax (tessellation.rs:482-495) */
void vdo_relax(vdo_tess* t) {
  size_t n = t->ncells < t->ngen ? t->ncells : t->ngen;
  double* ng = (double*)malloc((n ? n : 1) * 3 * sizeof(double));
  for (size_t i = 0; i < n; ++i) {
    if (t->cells[i].nv == 0) memcpy(&ng[3 * i], &t->gen[3 * i], 3 * sizeof(double));
    else cell_measure(&t->cells[i], NULL, &ng[3 * i], NULL);
  }
  vdo_set_generators(t, ng, n);
  free(ng);
}

/* one wall's WallGeometry::contains / cut (the cut's planes into p, n; returns
   their count), for the tests of the library's host-side wall queries */
int vdo_wall_contains_at(const vdo_tess* t, int w, const double p[3]) { return wall_contains(&t->walls[w], p); }
int vdo_wall_cut_at(const vdo_tess* t, int w, const double g[3], double* p, double* n) {
  return wall_cut(&t->walls[w], g, p, n);
}
size_t vdo_count_generators(const vdo_tess* t) { return t->ngen; }
void vdo_get_bins(const vdo_tess* t, size_t* start, size_t* members) {
  memcpy(start, t->bin_start, (t->nx * t->ny * t->nz + 1) * sizeof(size_t));
  memcpy(members, t->bin_members, t->ngen * sizeof(size_t));
}
size_t vdo_count_cells(const vdo_tess* t) { return t->ncells; }
void vdo_get_generators(const vdo_tess* t, double* xyz) { memcpy(xyz, t->gen, t->ngen * 3 * sizeof(double)); }
size_t vdo_search_order_len(const vdo_tess* t) { return t->norder; }
void vdo_get_search_order(const vdo_tess* t, int32_t* dxyz, double* min_d2) {
  for (size_t k = 0; k < t->norder; ++k) {
    if (dxyz) { dxyz[3 * k] = t->order[k].dx; dxyz[3 * k + 1] = t->order[k].dy; dxyz[3 * k + 2] = t->order[k].dz; }
    if (min_d2) min_d2[k] = t->order[k].min_d2;
  }
}

void vdo_get_summaries(const vdo_tess* t, double* vol, double* cen, int32_t* nfaces) {
  for (size_t i = 0; i < t->ncells; ++i) {
    double v, c[3];
    cell_measure(&t->cells[i], &v, c, NULL);
    if (vol) vol[i] = v;
    if (cen) { cen[3 * i] = c[0]; cen[3 * i + 1] = c[1]; cen[3 * i + 2] = c[2]; }
    if (nfaces) nfaces[i] = (int32_t)t->cells[i].nf;
  }
}

int64_t vdo_total_faces(const vdo_tess* t) {
  int64_t s = 0;
  for (size_t i = 0; i < t->ncells; ++i) s += (int64_t)t->cells[i].nf;
  return s;
}

void vdo_get_neighbors(const vdo_tess* t, int64_t* offsets, int32_t* ids) {
  int64_t o = 0;
  for (size_t i = 0; i < t->ncells; ++i) {
    if (offsets) offsets[i] = o;
    for (size_t f = 0; f < t->cells[i].nf; ++f) ids[o++] = t->cells[i].fn[f];
  }
  if (offsets) offsets[t->ncells] = o;
}

void vdo_get_face_areas(const vdo_tess* t, int64_t* offsets, double* areas) {
  int64_t o = 0;
  for (size_t i = 0; i < t->ncells; ++i) {
    const vdo_cell* c = &t->cells[i];
    if (offsets) offsets[i] = o;
    size_t off = 0;
    for (size_t f = 0; f < c->nf; ++f) {
      areas[o++] = face_area_at(c, off, c->fc[f]);
      off += c->fc[f];
    }
  }
  if (offsets) offsets[t->ncells] = o;
}

void vdo_get_counters(const vdo_tess* t, uint64_t* out) { memcpy(out, t->counters, sizeof(t->counters)); }

const vdo_cell* vdo_get_cell(const vdo_tess* t, size_t i) { return i < t->ncells ? &t->cells[i] : NULL; }

/* ---- single-cell API ---- */
vdo_cell* vdo_cell_new(size_t id, const double bmin[3], const double bmax[3]) {
  vdo_cell* c = (vdo_cell*)calloc(1, sizeof(vdo_cell));
  cell_init_box(c, id, bmin, bmax);
  return c;
}

vdo_cell* vdo_cell_clone(const vdo_cell* c) {
  vdo_cell* d = (vdo_cell*)calloc(1, sizeof(vdo_cell));
  d->id = c->id;
  GROW(d->v, d->cap_v, 3 * c->nv + 1); memcpy(d->v, c->v, 3 * c->nv * sizeof(double)); d->nv = c->nv;
  GROW(d->fc, d->cap_fc, c->nf + 1); memcpy(d->fc, c->fc, c->nf); d->nf = c->nf;
  GROW(d->fn, d->cap_fn, c->nf + 1); memcpy(d->fn, c->fn, c->nf * sizeof(int32_t));
  GROW(d->fi, d->cap_fi, c->nh + 1); memcpy(d->fi, c->fi, c->nh * sizeof(uint16_t)); d->nh = c->nh;
  return d;
}

void vdo_cell_free(vdo_cell* c) {
  if (!c) return;
  free(c->v); free(c->fc); free(c->fn); free(c->fi); free(c);
}

int vdo_cell_clip(vdo_cell* c, const double point[3], const double normal[3], int neighbor_id) {
  scratch_t s;
  memset(&s, 0, sizeof(s));
  double r2;
  int m = cell_clip(c, point, normal, neighbor_id, &s, NULL, &r2, NULL);
  scratch_free(&s);
  return m;
}

int vdo_cell_num_vertices(const vdo_cell* c) { return (int)c->nv; }
int vdo_cell_num_faces(const vdo_cell* c) { return (int)c->nf; }
int vdo_cell_num_face_indices(const vdo_cell* c) { return (int)c->nh; }
size_t vdo_cell_id(const vdo_cell* c) { return c->id; }

void vdo_cell_export(const vdo_cell* c, double* verts, uint32_t* face_counts,
                     uint32_t* face_indices, int32_t* face_neighbors) {
  if (verts) memcpy(verts, c->v, 3 * c->nv * sizeof(double));
  for (size_t f = 0; f < c->nf; ++f) {
    if (face_counts) face_counts[f] = c->fc[f];
    if (face_neighbors) face_neighbors[f] = c->fn[f];
  }
  if (face_indices)
    for (size_t h = 0; h < c->nh; ++h) face_indices[h] = c->fi[h];
}

double vdo_cell_volume(const vdo_cell* c) { double v; cell_measure(c, &v, NULL, NULL); return v; }
void vdo_cell_centroid(const vdo_cell* c, double out[3]) { cell_measure(c, NULL, out, NULL); }
double vdo_cell_max_radius_sq(const vdo_cell* c, const double center[3]) { return cell_max_radius_sq(c, center); }

double vdo_cell_face_area(const vdo_cell* c, size_t face) {
  if (face >= c->nf) return 0.0;
  size_t off = 0;
  for (size_t f = 0; f < face; ++f) off += c->fc[f];
  return face_area_at(c, off, c->fc[face]);
}
