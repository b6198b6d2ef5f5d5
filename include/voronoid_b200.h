/*
 * voronoid_b200.h -- C ABI of the B200 tessellation library.
 *
 * A GPU-backed drop-in for the reference crate `voronoid`'s 3D path:
 * Tessellation<3, Cell3DFaces, Algorithm3DGrid> with plane, sphere, cylinder,
 * cone, torus and convex-polyhedron walls.
 * Every entry point below names the reference interface it replaces
 * (file:line within the reference crate).  Plain pointers and sizes only; no
 * framework types cross this boundary.
 *
 * Conventions
 *  - Every call returns an int status (VD_OK on success); the message of the
 *    last failure on a handle is available from vd_last_error().
 *  - A handle owns its device buffers and one CUDA stream.  A handle is not
 *    thread-safe (the reference's calculate takes &mut self); distinct
 *    handles may be used from different threads concurrently.
 *  - Host output buffers are owned by the caller and sized by query calls.
 *  - There is no CPU fallback: without a usable CUDA device every compute
 *    call returns VD_ECUDA.
 */
#ifndef VORONOID_B200_H
#define VORONOID_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define VD_OK 0
#define VD_EINVAL 1     /* bad argument; e.g. wall id > -1000 (reference panics, wall/mod.rs:25-27) */
#define VD_ENOMEM 2     /* device allocation failed or HBM budget exceeded */
#define VD_EOVERFLOW 3  /* a cell exceeded every polytope capacity (65534 vertices, 32767
                           faces; the standalone vd_cell: 2048 vertices, 512 faces) */
#define VD_ETIMEOUT 4   /* a bounded device wait gave up */
#define VD_ECUDA 5      /* CUDA runtime error / no device */
#define VD_ESTATE 6     /* call out of order (e.g. results before calculate) */
#define VD_EIO 7        /* a file could not be read (import_generators) */
#define VD_ECANCELED 8  /* a served request was cancelled before it started */

/* precision of the clipping path */
#define VD_PREC_FP64 0  /* plain FP64, bitwise the reference's arithmetic */
#define VD_PREC_MIXED 1 /* FP32 classification under an error bound, FP64 construction */

/* layout of the shared-memory tier's polytope (a tuning choice; results are
 * identical): slots rewrite only the faces a clip cuts (default), full
 * rewrites every face loop on each modifying clip, as the reference does */
#define VD_FAST_SLOTS 0
#define VD_FAST_FULL 1

/* WALL_ID_MAX (wall/mod.rs:8) */
#define VD_WALL_ID_MAX (-1000)

typedef struct vd_tess vd_tess;

/* ---- Tessellation::new + Algorithm3DGrid::new
 *      (tessellation.rs:25-36, algo_3d_grid.rs:47-95) ---- */
/* Errors: VD_EINVAL for a grid resolution outside [1, 16000] or a box whose
 * extent is not positive and finite on every axis (the reference's grid scale
 * n / (max - min) would be infinite or NaN); VD_ECUDA without a device. */
int vd_tess_create(const double bmin[3], const double bmax[3], int nx, int ny, int nz,
                   vd_tess** out);
/* drop of Tessellation */
int vd_tess_destroy(vd_tess* t);
/* a fresh Tessellation::new on an existing handle (new bounds and grid, no
 * walls, no generators) that keeps the handle's device buffers */
int vd_tess_reset(vd_tess* t, const double bmin[3], const double bmax[3], int nx, int ny, int nz);
/* message of the last failed call on t (or of the last failed create when t is NULL) */
const char* vd_last_error(const vd_tess* t);

/* ---- walls: Wall::new + PlaneGeometry/SphereGeometry + Tessellation::add_wall
 *      (wall/mod.rs:24-32, wall_3d.rs:23-27,66-68, tessellation.rs:197-200).
 *      Adding a wall prunes generators outside it (tessellation.rs:175-194).
 *      At most 16 walls per tessellation (the kernels take them as a fixed
 *      table in their parameters; the reference's Vec has no bound): one more
 *      returns VD_EINVAL and changes nothing. ---- */
int vd_tess_add_wall_plane(vd_tess* t, const double point[3], const double normal[3], int id);
int vd_tess_add_wall_sphere(vd_tess* t, const double center[3], double radius, int id);
/* CylinderGeometry (wall_3d.rs:107-174): inside an infinite cylinder; the
 * axis is normalised as the reference's constructor does */
int vd_tess_add_wall_cylinder(vd_tess* t, const double center[3], const double axis[3], double radius, int id);
/* ConeGeometry (wall_3d.rs:177-262): inside an infinite cone with apex `tip`,
 * axis pointing into the cone, half-angle in radians */
int vd_tess_add_wall_cone(vd_tess* t, const double tip[3], const double axis[3], double angle, int id);
/* TorusGeometry (wall_3d.rs:265-365): inside the tube of a torus */
int vd_tess_add_wall_torus(vd_tess* t, const double center[3], const double axis[3], double major_radius,
                           double minor_radius, int id);
/* ConvexPolyhedronGeometry::new (wall_3d.rs:462-492, 690-708): the
 * intersection of half-spaces given as planes (point, normal pointing OUT of
 * the valid region), points and normals AoS [nplanes * 3]; at most 256
 * planes over all polyhedron walls of a tessellation */
int vd_tess_add_wall_polyhedron(vd_tess* t, const double* points, const double* normals, int nplanes, int id);
/* Tessellation::clear_walls (tessellation.rs:203-205) */
int vd_tess_clear_walls(vd_tess* t);

/* ---- generators ---- */
/* Tessellation::set_generators (tessellation.rs:43-67): keep points inside all
 * walls, in order, then bin them (algo_3d_grid.rs:111-130). xyz is AoS, host. */
int vd_tess_set_generators(vd_tess* t, const double* xyz, size_t n, size_t* n_kept);
/* same, from a device pointer (the caller's CUDA memory, read on t's stream) */
int vd_tess_set_generators_device(vd_tess* t, const double* d_xyz, size_t n, size_t* n_kept);
/* Tessellation::set_generator (tessellation.rs:71-92): ignored when out of
 * range or outside a wall, as in the reference */
int vd_tess_set_generator(vd_tess* t, size_t index, const double xyz[3]);
/* Tessellation::random_generators (tessellation.rs:96-121), seeded: candidate
 * a = 0, 1, ... has coordinates min[c] + u * (max[c] - min[c]) with
 * u = (splitmix64 draw 3a + c of `seed`) >> 11, times 2^-53; the first `count`
 * candidates inside every wall become the generators, out of at most
 * count * 1000 attempts (*n_found may then be below count).  The reference
 * seeds from thread_rng; a caller wanting that passes a random seed. */
int vd_tess_random_generators(vd_tess* t, size_t count, uint64_t seed, size_t* n_found);
/* Tessellation::read_generators (tessellation.rs:153-171): one generator per
 * line of `text` (len bytes of UTF-8): an id, ignored, then x y z; a missing
 * or unparsable coordinate reads 0.0 (Rust's str::parse::<f64> grammar), a
 * line with no token is skipped.  The points then go through set_generators.
 * VD_EINVAL, with nothing changed, when the bytes are not UTF-8 (a Rust &str
 * always is). */
int vd_tess_read_generators(vd_tess* t, const char* text, size_t len, size_t* n_kept);
/* Tessellation::import_generators (tessellation.rs:126-148): the same for a
 * file; VD_EIO when it cannot be read, VD_EINVAL when it is not UTF-8 (the
 * reference returns the io::Error); nothing is changed then. */
int vd_tess_import_generators(vd_tess* t, const char* path, size_t* n_kept);
/* the parser of vd_tess_read_generators alone (host only, no device): writes
 * min(cap, *n_points) points (AoS) to xyz; *n_points = points in the text.
 * Errors: VD_EINVAL (message via vd_last_error(NULL)). */
int vd_parse_generators(const char* text, size_t len, double* xyz, size_t cap, size_t* n_points);
/* Tessellation::count_generators / generators (tessellation.rs:498-500,519-521) */
int vd_tess_count_generators(const vd_tess* t, size_t* n);
int vd_tess_get_generators(vd_tess* t, double* xyz);

/* ---- the hot path ---- */
/* select VD_PREC_FP64 (default) or VD_PREC_MIXED for the next calculate */
int vd_tess_set_precision(vd_tess* t, int precision);
/* select VD_FAST_SLOTS (default) or VD_FAST_FULL for the next calculate (no
 * counterpart in the reference: a layout choice of this library's first
 * tier, made by the autotuner; every choice gives the same results) */
int vd_tess_set_fast_layout(vd_tess* t, int layout);

/* Launch choices the autotuner makes (no counterpart in the reference; every
 * setting gives the same results bit for bit, only the time changes).  A
 * field of 0 keeps the library's default. */
typedef struct {
  int fast_layout;         /* VD_FAST_SLOTS (default) or VD_FAST_FULL */
  int fast_blocks_per_sm;  /* slot layout: 5, 6 or 7 blocks of four warps per SM (default 7 for FP64, 6 for
                              mixed precision; vd_tess_get_tuning reports the one in force) (the register budget
                              of the compiled variant; the shared-memory tier's polytopes always fit) */
  int huge_direct_max;     /* cells left after the medium tier, at most this many (default 64) go straight to
                              the block-per-cell tier instead of through the large tier */
  int huge_blocks_max;     /* most concurrent blocks of the block-per-cell tier (default 64, at most 256) */
  int huge_narrow_max;     /* tessellations of at most this many cells run that tier with 16-warp blocks,
                              larger ones with 32 (default 2^30: always 16) */
  int noop_run;            /* after this many clips in a row that changed nothing, the walk tests the next
                              candidates' planes together, one per lane, and passes over those that cut
                              nothing (-1: never; 0 keeps the default, -1) */
} vd_tuning;
int vd_tess_set_tuning(vd_tess* t, const vd_tuning* k);
/* the settings in force (defaults filled in) */
int vd_tess_get_tuning(const vd_tess* t, vd_tuning* k);
/* Tessellation::calculate (tessellation.rs:213-230) over compute_cell
 * (:414-475), Algorithm3DGrid::visit_neighbors (algo_3d_grid.rs:145-202) and
 * Cell3DFaces::clip_with_scratch (cell_3d_faces.rs:288-503), with the volume,
 * centroid and face-area reductions (cell_3d_faces.rs:106-254) fused in. */
int vd_tess_calculate(vd_tess* t);
/* The same computation restricted to the cells with ids in [begin, end): the
 * shard of one process when a tessellation's cells are split across GPUs
 * (each GPU holds all generators and computes its own id range).  Cells
 * outside the range read as empty (volume 0, centroid 0, no faces), as in
 * the reference's per-cell map (tessellation.rs:223-229) restricted to the
 * range.  VD_EINVAL unless begin <= end <= count_generators. */
int vd_tess_calculate_range(vd_tess* t, size_t begin, size_t end);
/* The same over interleaved chunks (no counterpart in the reference): the
 * cells with ids in [begin, end) and ((id - begin) / chunk) % stride == phase.
 * With stride = the number of GPUs and phase = this GPU's rank, each GPU gets
 * an equal share of every part of the id order, so inputs whose cost varies
 * along the id order (clustered generators first, background after) balance
 * across GPUs.  VD_EINVAL unless chunk >= 1 and phase < stride.  A polytope
 * export (vd_tess_export_cells) needs a contiguous calculate: VD_ESTATE
 * after a strided one. */
int vd_tess_calculate_strided(vd_tess* t, size_t begin, size_t end, size_t chunk, size_t stride, size_t phase);
/* Tessellation::calculate_sealed (tessellation.rs:234-318): calculate, then
 * every cell on a curved wall (sphere, cylinder, cone, torus) is clipped with
 * the wall's tangent plane at each face neighbour on the same wall, when its
 * own generator lies on that plane's valid side.  Fills the seal log. */
int vd_tess_calculate_sealed(vd_tess* t);
/* Tessellation::prune_boundaries (tessellation.rs:323-385): for every cell on
 * a curved wall and every distinct neighbour on the same wall, the vertices
 * the cell's wall faces share with its faces towards that neighbour
 * (Cell::shared_vertices, cell_3d_faces.rs:536-565).  Fills the prune logs;
 * the cells are unchanged. */
int vd_tess_prune_boundaries(vd_tess* t);
/* seal_log (tessellation.rs:19): (cell, neighbour, wall id) per seal clip
 * that changed a cell, in cell order; *n = number of int32 values.  Call
 * with out = NULL for the size.  Cleared by calculate. */
int vd_tess_seal_log(vd_tess* t, int32_t* out, size_t* n);
/* prune_log / prune_pos_log (tessellation.rs:20-21): (cell, neighbour, wall
 * id, vertex count) per entry and the vertices' xyz; *n_entries and
 * *n_positions count int32 and double values.  NULL buffers query sizes. */
int vd_tess_prune_log(vd_tess* t, int32_t* entries, size_t* n_entries, double* positions, size_t* n_positions);
/* Tessellation::relax (tessellation.rs:482-495), on the device */
int vd_tess_relax(vd_tess* t);
/* Tessellation::count_cells (tessellation.rs:503-505) */
int vd_tess_count_cells(const vd_tess* t, size_t* n);

/* ---- results (host buffers) ----
 * Per-cell summaries: Cell3DFaces::volume / centroid (cell_3d_faces.rs:106-205)
 * and the face count; any pointer may be NULL. */
int vd_tess_get_cell_summaries(vd_tess* t, double* volume, double* centroid3, int32_t* n_faces);
/* total faces over all cells (size of the CSR payloads below) */
int vd_tess_total_faces(vd_tess* t, int64_t* total);
/* Cell3DFaces::face_neighbors (cell_3d_faces.rs:97-99) of every cell as CSR:
 * offsets[n_cells+1], ids[total]; offsets may be NULL */
int vd_tess_get_neighbors(vd_tess* t, int64_t* offsets, int32_t* ids);
/* Cell3DFaces::face_area for every face of every cell (cell_3d_faces.rs:207-254) */
int vd_tess_get_face_areas(vd_tess* t, int64_t* offsets, double* areas);
/* Tessellation::get_cell (tessellation.rs:514-516): the full polytope of cell i
 * in the layout of Cell3DFaces (cell_3d_faces.rs:24-34).  Call with NULL
 * buffers to get the sizes, then again with buffers of those sizes. */
int vd_tess_get_cell(vd_tess* t, size_t i, int32_t* n_vertices, int32_t* n_faces,
                     int32_t* n_face_indices, double* vertices, uint32_t* face_counts,
                     uint32_t* face_indices, int32_t* face_neighbors);

/* Tessellation::cells / map (tessellation.rs:391-412, 524-526) in bulk: the
 * Cell3DFaces of cells [begin, end) as CSR arrays.  v_off, f_off, h_off
 * [end - begin + 1] always get the offsets of each cell's vertices, faces and
 * face entries (cells outside the last calculate_range read as empty).  With
 * vertices [3 * v_off[n]], face_counts and face_neighbors [f_off[n]] and
 * face_indices [h_off[n]] given (all four, or none for the sizes only), each
 * cell's polytope is written at its offsets, exactly as vd_tess_get_cell gives
 * it; face_indices are local to the cell.  Device memory grows with the range:
 * export a large tessellation in ranges. */
int vd_tess_export_cells(vd_tess* t, size_t begin, size_t end, int64_t* v_off, int64_t* f_off, int64_t* h_off,
                         double* vertices, uint32_t* face_counts, uint32_t* face_indices, int32_t* face_neighbors);

/* ---- device-resident results (for callers that keep data on the GPU) ---- */
int vd_tess_device_results(vd_tess* t, const double** d_volume, const double** d_centroid3,
                           const int32_t** d_n_faces);
/* the neighbour-id and face-area CSR (as vd_tess_get_neighbors /
 * vd_tess_get_face_areas give it) in device memory owned by t:
 * d_offsets[n_cells + 1], d_ids[*total], d_areas[*total]; valid until the next
 * call that changes t; the data is complete when the call returns */
int vd_tess_device_neighbors(vd_tess* t, const int64_t** d_offsets, const int32_t** d_ids, const double** d_areas,
                             int64_t* total);

/* ---- instrumentation ---- */
/* the CUDA stream (cudaStream_t) all work of t is ordered on */
int vd_tess_stream(vd_tess* t, void** stream);
/* device time (ms, CUDA events) of the phases of the last calculate:
 * [0] binning, [1] clip kernel, [2] overflow/fallback passes, [3] total */
int vd_tess_timings(vd_tess* t, float* ms4);
/* run calculate with the instrumented kernel variant (off by default; the
 * counters cost a few percent of the clip kernel's time) */
int vd_tess_set_instrumentation(vd_tess* t, int on);
/* algorithmic event counters of the last instrumented calculate (same
 * meaning as the oracle's): candidates, clips, classified, modifying,
 * intersections, kept, triangles, offsets; VD_ESTATE when not instrumented */
int vd_tess_counters(vd_tess* t, uint64_t* out8);
/* cells that needed a fallback pass in the last calculate:
 * [0] polytope-capacity overflow, [1] search-order extension */
int vd_tess_fallback_counts(vd_tess* t, uint64_t* out2);

/* kernels this library has launched in this process, over all handles */
int vd_launch_count(uint64_t* n);

/* ---- one cell on its own: Cell3DFaces (cell_3d_faces.rs:22-270) behind the
 *      Cell trait (cell/mod.rs:8-43) ----
 * The polytope lives in device memory (up to 2048 vertices, 512 faces, 6144
 * face entries) and every operation runs the tessellation kernels' own warp
 * routines, one small launch per call.  A handle is not thread-safe. */
typedef struct vd_cell vd_cell;
/* message of the last failed call on c (of the last failed create when c is NULL) */
const char* vd_cell_last_error(const vd_cell* c);
/* Cell3DFaces::new(id, bounds) (cell_3d_faces.rs:37-74): the box cell */
int vd_cell_create_box(size_t id, const double bmin[3], const double bmax[3], vd_cell** out);
/* a cell holding a given polytope in the Cell3DFaces layout (cell_3d_faces.rs:24-34),
 * e.g. one exported by vd_tess_get_cell; VD_EINVAL when a face entry names a
 * missing vertex or the polytope exceeds the capacities */
int vd_cell_create(size_t id, int32_t n_vertices, int32_t n_faces, const double* vertices,
                   const uint32_t* face_counts, const uint32_t* face_indices, const int32_t* face_neighbors,
                   vd_cell** out);
int vd_cell_destroy(vd_cell* c);
/* Cell3DFaces::id (cell_3d_faces.rs:77-79) */
int vd_cell_id(const vd_cell* c, size_t* id);
/* Cell::clip = Cell3DFaces::clip_with_scratch (cell_3d_faces.rs:288-503):
 * clip by the plane (point, normal); the kept side is (v - point).normal <= 1e-9
 * and the new face gets neighbor_id.  *modified and *max_radius_sq are the
 * reference's returned (bool, f64): the max squared distance of the new
 * vertices from `generator`, 0 when generator is NULL or nothing changed. */
int vd_cell_clip(vd_cell* c, const double point[3], const double normal[3], int32_t neighbor_id,
                 const double* generator, int* modified, double* max_radius_sq);
/* Cell3DFaces::max_radius_sq (cell_3d_faces.rs:271-286) */
int vd_cell_max_radius_sq(vd_cell* c, const double center[3], double* out);
/* volume, centroid, face count, and the area and neighbour of every face
 * (cell_3d_faces.rs:106-254, 97-99); face_areas / face_neighbors hold
 * n_faces entries (call once with NULL to learn n_faces); any pointer may be NULL */
int vd_cell_measure(vd_cell* c, double* volume, double centroid3[3], int32_t* n_faces, double* face_areas,
                    int32_t* face_neighbors);
/* the polytope (vertices, face_counts, face_indices, face_neighbors); call
 * with NULL buffers to get the sizes */
int vd_cell_get(vd_cell* c, int32_t* n_vertices, int32_t* n_faces, int32_t* n_face_indices, double* vertices,
                uint32_t* face_counts, uint32_t* face_indices, int32_t* face_neighbors);

/* ---- pinned host memory for callers staging large inputs/outputs ---- */
int vd_host_alloc(size_t bytes, void** ptr);
int vd_host_free(void* ptr);

/* ---- batches: many independent tessellations in one persistent launch ----
 * Each member is a Tessellation with its own bounds, grid, walls and
 * generators and computes exactly what a vd_tess with the same inputs
 * computes; the batch only shares the launches (no counterpart in the
 * reference, which computes one tessellation per call). */
typedef struct vd_batch vd_batch;
/* a wall of a batch member or a served request (the geometries of
 * wall_3d.rs, normalised as their constructors do):
 *   kind 0 PlaneGeometry      a = point, n = normal into the valid region
 *   kind 1 SphereGeometry     a = centre, r = radius
 *   kind 2 CylinderGeometry   a = centre, n = axis, r = radius
 *   kind 3 ConeGeometry       a = tip, n = axis (into the cone), r = half-angle (radians)
 *   kind 4 TorusGeometry      a = centre, n = axis, r = major radius, r2 = minor radius
 *   kind 5 ConvexPolyhedronGeometry  points / normals [3 * nplanes], normals pointing out
 * id <= VD_WALL_ID_MAX; the plane arrays are copied by the call that takes the wall */
typedef struct {
  int kind;
  int id;
  double a[3];
  double n[3];
  double r;
  double r2;
  const double* points;
  const double* normals;
  int nplanes;
} vd_wall_desc;

/* ---- one wall, one grid, on the host (no device) ---- */
/* Wall::contains (wall/mod.rs:38-40; each geometry's contains, wall_3d.rs:31-36,
 * 73-78, 132-143, 202-214, 293-309, 691-701) for a wall described as for
 * batches: *inside = 1 or 0.  VD_EINVAL for a bad descriptor. */
int vd_wall_contains(const vd_wall_desc* wall, const double point[3], int* inside);
/* Wall::cut (wall/mod.rs:42-44; wall_3d.rs:38-42, 80-100, 145-173, 216-261,
 * 311-364, 703-708): the planes the wall emits for one generator, in the
 * order the reference's callback receives them (point, normal pointing out of
 * the valid region); *n = their count (0 or 1, or the polyhedron's planes),
 * min(*n, cap) written.  Bit for bit the planes the clip kernels use. */
int vd_wall_cut(const vd_wall_desc* wall, const double generator[3], double* points, double* normals, int cap,
                int* n);
/* Algorithm3DGrid::new's search order (algo_3d_grid.rs:56-76) as the kernels
 * use it: the offsets of [-k, k]^3 (clipped to the grid) sorted by min_d2, ties
 * in enumeration order; a table with k below the grid's size keeps the
 * offsets with min_d2 < *bound and sets *complete = 0.  *n = its length,
 * min(*n, cap) entries written (dxyz: 3 per entry). */
int vd_search_order(const double bmin[3], const double bmax[3], int nx, int ny, int nz, int k, int32_t* dxyz,
                    double* min_d2, size_t cap, size_t* n, int* complete, double* bound);
/* Algorithm3DGrid::get_bin_index (algo_3d_grid.rs:97-107) of the grid
 * Algorithm3DGrid::new(nx, ny, nz, bounds) builds */
int vd_grid_bin_index(const double bmin[3], const double bmax[3], int nx, int ny, int nz, const double point[3],
                      size_t* index);

int vd_batch_create(vd_batch** out);
int vd_batch_destroy(vd_batch* b);
const char* vd_batch_last_error(const vd_batch* b);
/* add a member: Tessellation::new + add_wall(s) + set_generators (host AoS);
 * *index receives its position in the batch */
int vd_batch_add(vd_batch* b, const double bmin[3], const double bmax[3], int nx, int ny, int nz,
                 const vd_wall_desc* walls, int nwalls, const double* xyz, size_t n, int* index);
int vd_batch_set_precision(vd_batch* b, int precision);
/* VD_FAST_SLOTS (default) or VD_FAST_FULL, as vd_tess_set_fast_layout */
int vd_batch_set_fast_layout(vd_batch* b, int layout);
int vd_batch_set_instrumentation(vd_batch* b, int on);
/* drop the members so that the batch takes new ones (vd_batch_add again);
 * device buffers are kept and only grow */
int vd_batch_reset(vd_batch* b);
/* upload every member and bin it (after the last vd_batch_add) */
int vd_batch_commit(vd_batch* b);
/* Tessellation::calculate for every member, one persistent launch */
int vd_batch_calculate(vd_batch* b);
/* steps x (Tessellation::relax then calculate) for every member, on the
 * device; a step is captured once in a CUDA graph and replayed */
int vd_batch_lloyd(vd_batch* b, int steps);
int vd_batch_count(const vd_batch* b, int* ntess);
int vd_batch_count_cells(const vd_batch* b, int index, size_t* n);
int vd_batch_total_cells(const vd_batch* b, size_t* n);
int vd_batch_get_generators(vd_batch* b, int index, double* xyz);
int vd_batch_get_summaries(vd_batch* b, int index, double* volume, double* centroid3, int32_t* n_faces);
/* device time (ms) of the last calculate / lloyd call */
int vd_batch_timing(const vd_batch* b, float* ms);
int vd_batch_counters(const vd_batch* b, uint64_t* out8);
int vd_batch_stream(vd_batch* b, void** stream);

/* ---- serving: a request loop with continuous batching (no counterpart in
 * the reference) ----
 * `slots` worker threads each keep one resident tessellation handle with its
 * own CUDA stream.  Requests (one Tessellation job each) are admitted FIFO
 * as soon as a slot is free and their estimated device footprint fits in
 * hbm_budget_bytes beside the running ones; running requests overlap on the
 * device.  A request's result equals a standalone vd_tess's for the same
 * inputs. */
typedef struct vd_server vd_server;
int vd_server_create(int slots, size_t hbm_budget_bytes, int precision, vd_server** out);
int vd_server_destroy(vd_server* s);
const char* vd_server_last_error(const vd_server* s);
/* copies the inputs; *ticket identifies the request */
int vd_server_submit(vd_server* s, const double bmin[3], const double bmax[3], int nx, int ny, int nz,
                     const vd_wall_desc* walls, int nwalls, const double* xyz, size_t n, uint64_t* ticket);
/* the same with the generators as text in the read_generators format (see
 * vd_tess_read_generators), parsed on the submitting thread; the request's
 * latency includes the parse.  VD_EINVAL when the text is not UTF-8. */
int vd_server_submit_text(vd_server* s, const double bmin[3], const double bmax[3], int nx, int ny, int nz,
                          const vd_wall_desc* walls, int nwalls, const char* text, size_t len, uint64_t* ticket);
/* blocks until the request is done: its cell count and submit-to-done latency */
int vd_server_wait(vd_server* s, uint64_t ticket, size_t* n_cells, double* latency_s);
/* copies the per-cell results (any pointer may be NULL) and releases the request */
int vd_server_take(vd_server* s, uint64_t ticket, double* volume, double* centroid3, int32_t* n_faces);
/* completed requests, their cells, latency p50/p99 (s), peak admitted bytes */
int vd_server_stats(vd_server* s, uint64_t* completed, uint64_t* cells, double* p50_s, double* p99_s,
                    size_t* peak_bytes);
int vd_server_reset_stats(vd_server* s);
/* requests on the GPU now and the most at once since the last reset_stats */
int vd_server_concurrency(vd_server* s, int* running, int* peak_running);
/* on = 1: requests submitted afterwards also return each cell's neighbour
 * ids and face areas (Cell3DFaces::face_neighbors / face_area,
 * cell_3d_faces.rs:97-99,207-254) as a CSR over cells (vd_server_take_faces) */
int vd_server_set_face_results(vd_server* s, int on);
/* blocks until the request is done; *total = its faces over all cells (the
 * size of the CSR arrays), 0 for a request submitted without face results */
int vd_server_total_faces(vd_server* s, uint64_t ticket, int64_t* total);
/* vd_server_take plus the CSR: offsets[n_cells + 1], ids[total], areas[total]
 * (any pointer may be NULL); releases the request */
int vd_server_take_faces(vd_server* s, uint64_t ticket, double* volume, double* centroid3, int32_t* n_faces,
                         int64_t* offsets, int32_t* ids, double* areas);
/* a request still in the queue is dropped (its wait/take return VD_ECANCELED);
 * one that has started runs to completion and this returns VD_ESTATE */
int vd_server_cancel(vd_server* s, uint64_t ticket);
/* merging of small requests (off by default; limits 65,536 generators a
 * request and 2^20 a group unless given): a slot that starts a request without face results
 * of at most max_request generators also takes the run of such requests
 * behind it in the queue (up to max_members, max_group generators in all,
 * within the HBM budget) and computes them as one batch (vd_batch); each
 * result equals the request's standalone result.  max_members <= 1 turns it
 * off; a zero size keeps the current one. */
int vd_server_set_merging(vd_server* s, int max_members, size_t max_request, size_t max_group);
/* merged batches run and the requests they served, since the last reset_stats */
int vd_server_merge_stats(vd_server* s, uint64_t* groups, uint64_t* merged_requests);

/* ---- fault injection for tests (no counterpart in the reference) ----
 * the next `count` device allocations this library makes (in any thread)
 * fail as out of memory (VD_ENOMEM), as a full GPU would; 0 clears it */
int vd_debug_fail_allocations(int count);

/* ---- allocation-free variant (no counterpart in the reference) ----
 * set_generators + calculate for a small tessellation without any device
 * allocation, for callers that cannot call cudaMalloc: a plugin inside an
 * application that owns the GPU's memory and hands out fixed buffers, code
 * bound to a framework's memory pool, or a latency-critical loop that cannot
 * take the device-wide synchronisation an allocation can cause.  The caller
 * passes device buffers: d_xyz (n generators, AoS) and per-cell outputs
 * d_volume[n], d_centroid3[3n], d_n_faces[n].  All intermediate data lives in
 * one fixed __device__ array (about 8 MiB) that every GPU loading the library
 * holds until exit.  Limits: n <= 8192 generators and a grid whose complete
 * search order fits, (2nx+1)(2ny+1)(2nz+1) <= 68921 (e.g. 20x20x20); larger
 * requests return VD_EINVAL (message via vd_last_error(NULL)).  No walls.
 * Cells are built with at most 2048 vertices and 512 faces each: a cell
 * beyond that (e.g. the centre of generators on a sphere, adjacent to
 * thousands of others), which the regular entry points build in their
 * block-per-cell tier, makes the call return VD_EOVERFLOW.
 * Calls share the array: calls that overlap on the GPU race, so order them
 * (e.g. on one stream).  The first call on a device resolves the array's
 * device address; make that first call before any stream capture begins.
 * Each call waits for its work on `stream` to finish before it returns.
 * stream may be NULL (the default stream).  Every result equals
 * vd_tess_set_generators_device + vd_tess_calculate bit for bit. */
int vd_calculate_noalloc(const double bmin[3], const double bmax[3], int nx, int ny, int nz,
                         const double* d_xyz, size_t n, double* d_volume, double* d_centroid3,
                         int32_t* d_n_faces, void* stream);

/* ---- device measurement helper: FP64 / FP32 FMA-chain peak (TFLOP/s) ---- */
int vd_measure_fma_peak(int fp64, double* tflops);

#ifdef __cplusplus
}
#endif
#endif
