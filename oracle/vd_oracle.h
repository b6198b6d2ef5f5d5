/*
 * vd_oracle.h -- CPU oracle for the 3D tessellation path (TEST INFRASTRUCTURE).
 *
 * This is a plain-C restatement of the reference crate `voronoid` (Rust) for
 * the path Tessellation::calculate over Algorithm3DGrid + Cell3DFaces, with
 * plane, sphere, cylinder, cone, torus and convex-polyhedron walls.  It
 * exists only to check the CUDA product path and to time a CPU baseline;
 * nothing in the product links or calls it.
 *
 * Parity pins: the reference cannot be compiled here (it is Rust and no Rust
 * toolchain exists), so this restatement is pinned against the reference's
 * own known-answer tests and its Voro++ golden vectors
 * (tests/data/{face_counts,vertex_positions}), committed as fixtures under
 * tests/golden/.
 *
 * Deliberate, documented difference: Algorithm3DGrid::new sorts its search
 * order with Rust's sort_unstable_by (algo_3d_grid.rs:76), whose tie order is
 * not reproducible without Rust.  The oracle uses a STABLE sort of the same
 * z-outer / x-inner enumeration, and the CUDA path uses the same table.
 */
#ifndef VD_ORACLE_H
#define VD_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vdo_tess vdo_tess;
typedef struct vdo_cell vdo_cell;

/* counters for the algorithmic flop model (summed over cells) */
enum {
  VDO_CNT_CANDIDATES = 0,   /* visitor calls (tessellation.rs:446) */
  VDO_CNT_CLIPS,            /* clip calls, walls + neighbours */
  VDO_CNT_CLASSIFIED,       /* vertex-plane distance evaluations */
  VDO_CNT_MODIFYING,        /* clips that rebuilt the polytope */
  VDO_CNT_INTERSECTIONS,    /* intersection vertices created */
  VDO_CNT_KEPT,             /* kept vertices (radius evaluated) */
  VDO_CNT_TRIANGLES,        /* fan triangles in volume/centroid */
  VDO_CNT_OFFSETS,          /* search-order entries examined */
  VDO_NCOUNTERS
};

/* ---- tessellation (tessellation.rs + algo_3d_grid.rs) ---- */
vdo_tess* vdo_create(const double bmin[3], const double bmax[3], int nx, int ny, int nz);
/* the same with the search order truncated to offsets |d| <= k on each axis
 * (for grids whose complete (2n+1)^3 table does not fit in memory); the
 * cells of the last calculate whose walk ran off it are counted by
 * vdo_table_exhausted, and their results are then not the reference's */
vdo_tess* vdo_create_truncated(const double bmin[3], const double bmax[3], int nx, int ny, int nz, int k);
size_t vdo_table_exhausted(const vdo_tess* t);
void vdo_destroy(vdo_tess* t);
/* returns 0, or -1 if id > -1000 (the reference panics, wall/mod.rs:25) */
int vdo_add_wall_plane(vdo_tess* t, const double point[3], const double normal[3], int id);
int vdo_add_wall_sphere(vdo_tess* t, const double center[3], double radius, int id);
/* CylinderGeometry / ConeGeometry / TorusGeometry / ConvexPolyhedronGeometry
 * (wall_3d.rs:107-365, 462-708); axes are normalised as the reference does */
int vdo_add_wall_cylinder(vdo_tess* t, const double center[3], const double axis[3], double radius, int id);
int vdo_add_wall_cone(vdo_tess* t, const double tip[3], const double axis[3], double angle, int id);
int vdo_add_wall_torus(vdo_tess* t, const double center[3], const double axis[3], double major, double minor,
                       int id);
int vdo_add_wall_polyhedron(vdo_tess* t, const double* points, const double* normals, int nplanes, int id);
/* planes of ConvexPolyhedronGeometry::new_{tetrahedron,hexahedron,octahedron,
 * dodecahedron,icosahedron} (kind = face count 4/6/8/12/20); returns the count */
int vdo_regular_polyhedron(int kind, const double center[3], double radius, double* points, double* normals);
void vdo_clear_walls(vdo_tess* t);
size_t vdo_set_generators(vdo_tess* t, const double* xyz, size_t n);
void vdo_set_generator(vdo_tess* t, size_t index, const double xyz[3]);
size_t vdo_random_generators(vdo_tess* t, size_t count, uint64_t seed);
/* wall w's contains / cut (p, n get 3 * count doubles; count <= 64) */
int vdo_wall_contains_at(const vdo_tess* t, int w, const double p[3]);
int vdo_wall_cut_at(const vdo_tess* t, int w, const double g[3], double* p, double* n);
/* grid_bins as CSR: start[nbins + 1], members[count_generators] */
void vdo_get_bins(const vdo_tess* t, size_t* start, size_t* members);
void vdo_calculate(vdo_tess* t, int nthreads);
/* calculate only cells [begin, end) (a bounded sample for timing) */
void vdo_calculate_range(vdo_tess* t, size_t begin, size_t end, int nthreads);
void vdo_relax(vdo_tess* t);
/* Tessellation::calculate_sealed / prune_boundaries (tessellation.rs:234-385)
 * and their logs: seal (cell, neighbour, wall id) triples; prune (cell,
 * neighbour, wall id, vertex count) quadruples with the vertices' xyz */
void vdo_calculate_sealed(vdo_tess* t, int nthreads);
void vdo_prune_boundaries(vdo_tess* t);
size_t vdo_seal_log_len(const vdo_tess* t);
void vdo_get_seal_log(const vdo_tess* t, int32_t* out);
size_t vdo_prune_log_len(const vdo_tess* t);
void vdo_get_prune_log(const vdo_tess* t, int32_t* out);
size_t vdo_prune_pos_log_len(const vdo_tess* t);
void vdo_get_prune_pos_log(const vdo_tess* t, double* out);
size_t vdo_count_generators(const vdo_tess* t);
size_t vdo_count_cells(const vdo_tess* t);
void vdo_get_generators(const vdo_tess* t, double* xyz);
size_t vdo_search_order_len(const vdo_tess* t);
void vdo_get_search_order(const vdo_tess* t, int32_t* dxyz, double* min_d2);
size_t vdo_bin_index(const vdo_tess* t, double x, double y, double z);

/* per-cell summaries: volume, centroid (3), face count */
void vdo_get_summaries(const vdo_tess* t, double* vol, double* cen, int32_t* nfaces);
int64_t vdo_total_faces(const vdo_tess* t);
/* CSR over cells in index order: offsets[n+1], ids / areas [total faces] */
void vdo_get_neighbors(const vdo_tess* t, int64_t* offsets, int32_t* ids);
void vdo_get_face_areas(const vdo_tess* t, int64_t* offsets, double* areas);
void vdo_get_counters(const vdo_tess* t, uint64_t* out);
/* borrow cell i of the last calculate (owned by t) */
const vdo_cell* vdo_get_cell(const vdo_tess* t, size_t i);

/* ---- single cell (cell_3d_faces.rs) ---- */
vdo_cell* vdo_cell_new(size_t id, const double bmin[3], const double bmax[3]);
vdo_cell* vdo_cell_clone(const vdo_cell* c);
void vdo_cell_free(vdo_cell* c);
/* clip_with_scratch with generator None; returns modified flag */
int vdo_cell_clip(vdo_cell* c, const double point[3], const double normal[3], int neighbor_id);
int vdo_cell_num_vertices(const vdo_cell* c);
int vdo_cell_num_faces(const vdo_cell* c);
int vdo_cell_num_face_indices(const vdo_cell* c);
void vdo_cell_export(const vdo_cell* c, double* verts, uint32_t* face_counts,
                     uint32_t* face_indices, int32_t* face_neighbors);
double vdo_cell_volume(const vdo_cell* c);
void vdo_cell_centroid(const vdo_cell* c, double out[3]);
double vdo_cell_face_area(const vdo_cell* c, size_t face);
double vdo_cell_max_radius_sq(const vdo_cell* c, const double center[3]);
size_t vdo_cell_id(const vdo_cell* c);

#ifdef __cplusplus
}
#endif
#endif
