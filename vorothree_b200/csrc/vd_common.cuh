// vd_common.cuh -- device-side data layout shared by the tessellation kernels.
//
// One tessellation on the device (HBM):
//   gen        double[3N]   generators, AoS, in the caller's order (index = cell id)
//   bin_of     u32[N]       bin of each generator (Algorithm3DGrid::generator_bin_ids)
//   bin_start  u32[B+1]     CSR of the bins; members ascending by generator id
//                           (Vec<Vec<usize>> grid_bins with push order, algo_3d_grid.rs:121-129)
//   sorted     SortedGen[N] generators in bin order (x, y, z, id), 32 B each, so a
//                           bin's members are one contiguous, aligned read
//   order      Offset[M]    shell search order (algo_3d_grid.rs:56-76), 16 B each
//   per-cell outputs: volume, centroid, face count, status, and per-face
//   neighbour ids and areas in fixed slots of FOUT faces per cell.
#pragma once
#include <cstdint>

namespace vd {

constexpr int kMaxWalls = 16;
constexpr double kTol = 1e-9;  // cell_3d_faces.rs:310-315,346,383-384

enum CellStatus : uint8_t {
  kCellOk = 0,
  kCellOverflow = 1,   // polytope exceeded the fast-path capacities
  kCellTable = 2,      // walked past the end of a truncated search order
  kCellHardFail = 3,   // exceeded even the large capacities
};

enum ClipResult : int { kClipNoop = 0, kClipMod = 1, kClipEmpty = 2, kClipOverflow = -1 };

enum Counter : int {
  kCntCandidates = 0,
  kCntClips,
  kCntClassified,
  kCntModifying,
  kCntIntersections,
  kCntKept,
  kCntTriangles,
  kCntOffsets,
  kNumCounters
};

struct Grid {
  double bmin[3], bmax[3];
  int n[3];
  double scale[3];  // grid_scale = n / extent
  double limit[3];  // grid_limit = n - 1e-5
  double cs[3];     // cell size = 1 / grid_scale
};

enum WallKind : int { kWallPlane = 0, kWallSphere, kWallCylinder, kWallCone, kWallTorus, kWallPolyhedron };

struct Wall {
  int kind;     // WallKind
  int id;
  double a[3];  // plane point / sphere, cylinder, torus centre / cone tip
  double n[3];  // plane normal pointing into the valid region / cylinder, cone, torus axis (normalised)
  double r;     // sphere, cylinder radius / torus major radius / cone half-angle
  double r2;    // torus minor radius
  double ca, sa, ta;  // cone: cos, sin and tan of the half-angle, computed on the host as libm does
  int np, p0;   // convex polyhedron: its planes are [p0, p0 + np) of the plane table
};

// planes of convex-polyhedron walls: (point, normal pointing out), 6 doubles each
constexpr int kMaxWallPlanes = 256;

struct alignas(16) Offset {
  int16_t dx, dy, dz, pad;
  double min_d2;
};

struct alignas(32) SortedGen {
  double x, y, z;
  long long id;
};

// Everything a clip kernel needs for one tessellation.
struct TessDesc {
  Grid grid;
  int nwalls;
  Wall walls[kMaxWalls];
  const double* planes;  // plane table of convex-polyhedron walls (device)
  const Offset* order;
  int norder;
  int order_complete;   // 1 when order holds every offset of the grid
  double order_bound;   // truncated table: every missing entry has min_d2 >= this
  const double* gen;
  const uint32_t* bin_of;
  const uint32_t* bin_start;
  const uint32_t* occ;  // optional: bit b set when bin b has members (sparse grids)
  int noop_run;         // > 0: a run of this many clips that changed nothing batches the walk's
                        // plane tests (compute_cell); 0: never
  const SortedGen* sorted;
  uint32_t ncells;
  // outputs
  double* vol;
  double* cen;
  int32_t* nfaces;
  int32_t* nverts;     // vertex count (0 = empty cell, Cell::is_empty)
  int32_t* fnb;        // [ncells * fout]
  double* farea;       // [ncells * fout]
  uint8_t* status;
  int fout;
  // faces of cells with more than fout faces (large-capacity pass only)
  int32_t* pool_fnb;
  double* pool_farea;
  long long* pool_off;  // per cell; valid when nfaces > fout
  unsigned long long* pool_cursor;
  long long pool_cap;
};

// Work description of one launch of a clip kernel.
struct WorkList {
  const uint32_t* items;     // cell ids (batched: sorted positions); nullptr = all, in bin order
  uint32_t nitems;
  const uint32_t* nitems_dev;  // when set, the item count is read from device memory
  unsigned int* cursor;      // persistent-warp work counter
  uint32_t* ovf_list;        // cells that overflowed the capacities
  unsigned int* ovf_count;
  uint32_t* tab_list;        // cells that ran off a truncated search order
  unsigned int* tab_count;
  unsigned long long* counters;  // kNumCounters
  unsigned int* tess_flags;      // batched: per tessellation, set when a cell needs a longer search order
  // optional full-polytope export of a single cell (get_cell)
  double* ex_verts;
  uint32_t* ex_fc;
  uint32_t* ex_fi;
  int32_t* ex_fn;
  int32_t* ex_sizes;  // nv, nf, nh
  int ex_cap_v, ex_cap_f, ex_cap_h;
};

// The second pass of calculate_sealed and the pass of prune_boundaries
// (tessellation.rs:234-385).  Both rebuild a cell (compute_cell), re-apply
// the seal clips when the cells are sealed, then either finalize the cell
// (seal) or log the vertices its curved-wall faces share with its
// neighbours' faces (prune).
struct SealLogRec {   // one clip of calculate_sealed
  int32_t cell, seq, nbr, wall;
};
struct PruneRec {     // one (cell, neighbour, wall) entry of prune_boundaries
  int32_t cell, seq, nbr, wall, count, pseq;
};
struct PrunePos {     // one shared vertex of a prune entry
  int32_t cell, pseq;
  double x, y, z;
};

struct SealArgs {
  int mode;        // 1: seal and finalize; 2: prune (re-seal first when `sealed`)
  int sealed;      // the current cells were sealed
  uint32_t curved; // bit k: wall k is curved (not planar)
  int fout;
  // topology of the cells before sealing (calculate's result)
  const int32_t* s_nf;
  const int32_t* s_fnb;
  const long long* s_pool_off;
  const int32_t* s_pool_fnb;
  const uint32_t* s_mask;   // bit k: wall k's id is a curved wall among the cell's faces
  // topology of the current cells (prune)
  const int32_t* c_nf;
  const int32_t* c_fnb;
  const long long* c_pool_off;
  const int32_t* c_pool_fnb;
  const uint32_t* c_mask;
  // logs: records appended in any order, placed by (cell, seq) afterwards;
  // per-cell counts are written only when the cell completes
  SealLogRec* seal_rec;
  PruneRec* prune_rec;
  PrunePos* prune_pos;
  unsigned int* rec_cursor;  // [0] seal / prune records, [1] positions
  uint32_t rec_cap, pos_cap;
  int32_t* cnt;    // per cell: log entries
  int32_t* pcnt;   // per cell: prune positions
};

}  // namespace vd
