// vd_cell.cu -- one Cell3DFaces on the device, operated on call by call.
//
// The reference exposes the cell type on its own (cell_3d_faces.rs:22-270,
// trait Cell in cell/mod.rs:8-43): build a box cell, clip it by planes, read
// its volume, centroid, face areas and polytope.  A vd_cell holds one
// polytope in device memory in the large-capacity layout (up to 2048
// vertices, 512 faces, 6144 face entries) and runs every operation with the
// same warp routines the tessellation kernels use -- warp_clip for
// clip_with_scratch, finalize_cell for the measures -- so a cell built here
// and a cell of a tessellation carry the same bits.  Each call is one
// single-warp launch on the cell's own stream; this is the per-cell API, not
// the throughput path.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/voronoid_b200.h"
#include "vd_clip.cuh"
#include "vd_internal.h"

using namespace vd;

namespace vd_cell_impl {

using CellCfg = BigCfg;
using Poly = WarpPoly<CellCfg>;
using VId = CellCfg::VId;
using FId = CellCfg::FId;

// result block of a clip / measure, copied back after each call
struct CellOut {
  int clip_result;  // ClipResult
  int pad;
  double r2;
  double vol;
  double cen[3];
  int32_t nfaces, nverts, nh, status;
};

// Cell3DFaces::new (cell_3d_faces.rs:37-74)
__global__ void k_cell_box(Poly* P, PolyState* S, Grid g) {
  PolyState s;
  poly_init_box<CellCfg>(*P, s, g, 0.0, 0.0, 0.0);
  if (threadIdx.x < kNumCounters) P->cnt[threadIdx.x] = 0;
  if (threadIdx.x == 0) *S = s;
}

// a given polytope (vertices, face offsets, face entries, face neighbours)
__global__ void k_cell_load(Poly* P, PolyState* S, int nv, int nf, int nh, const double* verts,
                            const uint32_t* fstart, const uint32_t* fidx, const int32_t* fnb) {
  const unsigned lane = lane_id();
  for (int v = lane; v < nv; v += 32) {
    P->vx[v] = verts[3 * v];
    P->vy[v] = verts[3 * v + 1];
    P->vz[v] = verts[3 * v + 2];
  }
  for (int f = lane; f <= nf; f += 32) P->fs[0][f] = (uint16_t)fstart[f];
  for (int f = lane; f < nf; f += 32) {
    P->fn[0][f] = fnb[f];
    for (uint32_t h = fstart[f]; h < fstart[f + 1]; ++h) P->pf[0][h] = (FId)f;
  }
  for (int h = lane; h < nh; h += 32) P->fi[0][h] = (VId)fidx[h];
  if (lane < kNumCounters) P->cnt[lane] = 0;
  if (lane == 0) {
    PolyState s;
    s.nv = nv;
    s.nf = nf;
    s.nh = nh;
    s.cb = 0;
    s.umax = 0.0;
    *S = s;
  }
}

// Cell3DFaces::clip_with_scratch (cell_3d_faces.rs:288-503)
__global__ void k_cell_clip(Poly* P, PolyState* S, double px, double py, double pz, double nx, double ny,
                            double nz, int nbr, int with_gen, double gx, double gy, double gz, CellOut* out) {
  PolyState s = *S;
  double r2 = 0.0;
  const int r = warp_clip<CellCfg>(*P, s, px, py, pz, nx, ny, nz, nbr, with_gen != 0, gx, gy, gz, &r2);
  __syncwarp();
  if (threadIdx.x == 0) {
    if (r != kClipOverflow) *S = s;
    out->clip_result = r;
    out->r2 = r2;
  }
}

// max_radius_sq (cell_3d_faces.rs:271-286)
__global__ void k_cell_radius(const Poly* P, const PolyState* S, double cx, double cy, double cz, CellOut* out) {
  const PolyState s = *S;
  const double m = poly_max_radius_sq<CellCfg>(*P, s, cx, cy, cz);
  if (threadIdx.x == 0) out->r2 = m;
}

// volume, centroid and face areas (cell_3d_faces.rs:106-254), through the
// tessellation kernels' reduction with a one-cell descriptor
__global__ void k_cell_measure(Poly* P, const PolyState* S, CellOut* out, int32_t* fnb, double* farea) {
  const PolyState s = *S;
  TessDesc T;
  memset(&T, 0, sizeof(T));
  T.ncells = 1;
  T.vol = &out->vol;
  T.cen = out->cen;
  T.nfaces = &out->nfaces;
  T.nverts = &out->nverts;
  T.fnb = fnb;
  T.farea = farea;
  uint8_t st = 0;
  __shared__ uint8_t status;
  T.status = &status;
  T.fout = CellCfg::FCAP;
  finalize_cell<CellCfg>(T, 0, *P, s);
  __syncwarp();
  if (threadIdx.x == 0) {
    st = status;
    out->status = st;
    out->nh = s.nh;
  }
}

__global__ void k_cell_export(const Poly* P, const PolyState* S, WorkList W) {
  const PolyState s = *S;
  export_cell<CellCfg>(W, *P, s);
}

}  // namespace vd_cell_impl

using namespace vd_cell_impl;

struct vd_cell {
  std::string err;
  int device = 0;
  size_t id = 0;
  cudaStream_t stream = nullptr;
  Poly* poly = nullptr;
  PolyState* state = nullptr;
  CellOut* out = nullptr;
  int32_t* fnb = nullptr;
  double* farea = nullptr;
  // export staging: vertices, face counts, face entries, face neighbours, sizes
  double* ex_v = nullptr;
  uint32_t* ex_fc = nullptr;
  uint32_t* ex_fi = nullptr;
  int32_t* ex_fn = nullptr;
  int32_t* ex_sizes = nullptr;
  bool broken = false;  // a clip overflowed the capacities; the polytope is gone
};

namespace {

thread_local std::string g_cell_create_error;

int cfail(vd_cell* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  else g_cell_create_error = buf;
  return code;
}

#define VC_CK(c, call)                                                                              \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess)                                                                          \
      return cfail((c), e_ == cudaErrorMemoryAllocation ? VD_ENOMEM : VD_ECUDA, "%s: %s (%s:%d)", #call, \
                   cudaGetErrorString(e_), __FILE__, __LINE__);                                     \
  } while (0)

void release(vd_cell* c) {
  cudaFree(c->poly);
  cudaFree(c->state);
  cudaFree(c->out);
  cudaFree(c->fnb);
  cudaFree(c->farea);
  cudaFree(c->ex_v);
  cudaFree(c->ex_fc);
  cudaFree(c->ex_fi);
  cudaFree(c->ex_fn);
  cudaFree(c->ex_sizes);
  if (c->stream) cudaStreamDestroy(c->stream);
}

int alloc(vd_cell* c) {
  VC_CK(c, cudaGetDevice(&c->device));
  VC_CK(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  VC_CK(c, cudaMalloc(&c->poly, sizeof(Poly)));
  VC_CK(c, cudaMalloc(&c->state, sizeof(PolyState)));
  VC_CK(c, cudaMalloc(&c->out, sizeof(CellOut)));
  VC_CK(c, cudaMalloc(&c->fnb, CellCfg::FCAP * sizeof(int32_t)));
  VC_CK(c, cudaMalloc(&c->farea, CellCfg::FCAP * sizeof(double)));
  VC_CK(c, cudaMalloc(&c->ex_v, 3 * CellCfg::VCAP * sizeof(double)));
  VC_CK(c, cudaMalloc(&c->ex_fc, CellCfg::FCAP * sizeof(uint32_t)));
  VC_CK(c, cudaMalloc(&c->ex_fi, CellCfg::HCAP * sizeof(uint32_t)));
  VC_CK(c, cudaMalloc(&c->ex_fn, CellCfg::FCAP * sizeof(int32_t)));
  VC_CK(c, cudaMalloc(&c->ex_sizes, 4 * sizeof(int32_t)));
  return VD_OK;
}

int ready(vd_cell* c) {
  if (!c) return VD_EINVAL;
  if (c->broken) return cfail(c, VD_EOVERFLOW, "an earlier clip exceeded the cell's capacities");
  VC_CK(c, cudaSetDevice(c->device));
  return VD_OK;
}

int fetch_out(vd_cell* c, CellOut* h) {
  VC_CK(c, cudaMemcpyAsync(h, c->out, sizeof(CellOut), cudaMemcpyDeviceToHost, c->stream));
  VC_CK(c, cudaStreamSynchronize(c->stream));
  return VD_OK;
}

}  // namespace

extern "C" {

const char* vd_cell_last_error(const vd_cell* c) { return c ? c->err.c_str() : g_cell_create_error.c_str(); }

int vd_cell_create_box(size_t id, const double bmin[3], const double bmax[3], vd_cell** out) {
  if (!out || !bmin || !bmax) return cfail(nullptr, VD_EINVAL, "null argument");
  *out = nullptr;
  vd_cell* c = new vd_cell();
  c->id = id;
  int r = alloc(c);
  if (r != VD_OK) {
    g_cell_create_error = c->err;
    release(c);
    delete c;
    return r;
  }
  Grid g;
  memset(&g, 0, sizeof(g));
  for (int a = 0; a < 3; ++a) {
    g.bmin[a] = bmin[a];
    g.bmax[a] = bmax[a];
  }
  k_cell_box<<<1, 32, 0, c->stream>>>(c->poly, c->state, g);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    cfail(nullptr, VD_ECUDA, "cell setup: %s", cudaGetErrorString(e));
    release(c);
    delete c;
    return VD_ECUDA;
  }
  *out = c;
  return VD_OK;
}

int vd_cell_create(size_t id, int32_t n_vertices, int32_t n_faces, const double* vertices,
                   const uint32_t* face_counts, const uint32_t* face_indices, const int32_t* face_neighbors,
                   vd_cell** out) {
  if (!out) return cfail(nullptr, VD_EINVAL, "null argument");
  *out = nullptr;
  if (n_vertices < 0 || n_faces < 0 || n_vertices > CellCfg::VCAP || n_faces > CellCfg::FCAP)
    return cfail(nullptr, VD_EINVAL, "a cell holds at most %d vertices and %d faces", CellCfg::VCAP, CellCfg::FCAP);
  if ((n_vertices && !vertices) || (n_faces && (!face_counts || !face_neighbors)))
    return cfail(nullptr, VD_EINVAL, "null polytope array");
  std::vector<uint32_t> fstart((size_t)n_faces + 1, 0);
  for (int f = 0; f < n_faces; ++f) fstart[f + 1] = fstart[f] + face_counts[f];
  const uint32_t nh = fstart[n_faces];
  if (nh > (uint32_t)CellCfg::HCAP) return cfail(nullptr, VD_EINVAL, "a cell holds at most %d face entries", CellCfg::HCAP);
  if (nh && !face_indices) return cfail(nullptr, VD_EINVAL, "null face_indices");
  for (uint32_t h = 0; h < nh; ++h)
    if (face_indices[h] >= (uint32_t)n_vertices)
      return cfail(nullptr, VD_EINVAL, "face entry %u names vertex %u of %d", h, face_indices[h], n_vertices);
  vd_cell* c = new vd_cell();
  c->id = id;
  int r = alloc(c);
  double* d_v = nullptr;
  uint32_t *d_fs = nullptr, *d_fi = nullptr;
  int32_t* d_fn = nullptr;
  cudaError_t e = cudaSuccess;
  if (r == VD_OK) {
    e = cudaMalloc(&d_v, std::max<size_t>(1, 3 * (size_t)n_vertices) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_fs, fstart.size() * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&d_fi, std::max<size_t>(1, nh) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&d_fn, std::max<size_t>(1, (size_t)n_faces) * sizeof(int32_t));
    if (e == cudaSuccess && n_vertices)
      e = cudaMemcpyAsync(d_v, vertices, 3 * (size_t)n_vertices * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_fs, fstart.data(), fstart.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && nh)
      e = cudaMemcpyAsync(d_fi, face_indices, nh * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && n_faces)
      e = cudaMemcpyAsync(d_fn, face_neighbors, (size_t)n_faces * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
      k_cell_load<<<1, 32, 0, c->stream>>>(c->poly, c->state, n_vertices, n_faces, (int)nh, d_v, d_fs, d_fi, d_fn);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  }
  cudaFree(d_v);
  cudaFree(d_fs);
  cudaFree(d_fi);
  cudaFree(d_fn);
  if (r != VD_OK || e != cudaSuccess) {
    if (r == VD_OK) cfail(nullptr, VD_ECUDA, "cell setup: %s", cudaGetErrorString(e));
    else g_cell_create_error = c->err;
    release(c);
    delete c;
    return r != VD_OK ? r : VD_ECUDA;
  }
  *out = c;
  return VD_OK;
}

int vd_cell_destroy(vd_cell* c) {
  if (!c) return VD_OK;
  cudaSetDevice(c->device);
  release(c);
  delete c;
  return VD_OK;
}

int vd_cell_id(const vd_cell* c, size_t* id) {
  if (!c || !id) return VD_EINVAL;
  *id = c->id;
  return VD_OK;
}

int vd_cell_clip(vd_cell* c, const double point[3], const double normal[3], int32_t neighbor_id,
                 const double* generator, int* modified, double* max_radius_sq) {
  int r = ready(c);
  if (r != VD_OK) return r;
  if (!point || !normal) return cfail(c, VD_EINVAL, "null plane");
  const double* g = generator;
  k_cell_clip<<<1, 32, 0, c->stream>>>(c->poly, c->state, point[0], point[1], point[2], normal[0], normal[1],
                                        normal[2], neighbor_id, g ? 1 : 0, g ? g[0] : 0.0, g ? g[1] : 0.0,
                                        g ? g[2] : 0.0, c->out);
  VC_CK(c, cudaGetLastError());
  CellOut h;
  r = fetch_out(c, &h);
  if (r != VD_OK) return r;
  if (h.clip_result == kClipOverflow) {
    c->broken = true;
    return cfail(c, VD_EOVERFLOW, "clip exceeds the cell's capacities (%d vertices, %d faces)", CellCfg::VCAP,
                 CellCfg::FCAP);
  }
  // (modified, new max radius) as the reference's clip returns them
  if (modified) *modified = h.clip_result != kClipNoop;
  if (max_radius_sq) *max_radius_sq = h.clip_result == kClipMod ? h.r2 : 0.0;
  return VD_OK;
}

int vd_cell_max_radius_sq(vd_cell* c, const double center[3], double* out) {
  int r = ready(c);
  if (r != VD_OK) return r;
  if (!center || !out) return cfail(c, VD_EINVAL, "null argument");
  k_cell_radius<<<1, 32, 0, c->stream>>>(c->poly, c->state, center[0], center[1], center[2], c->out);
  VC_CK(c, cudaGetLastError());
  CellOut h;
  r = fetch_out(c, &h);
  if (r != VD_OK) return r;
  *out = h.r2;
  return VD_OK;
}

int vd_cell_measure(vd_cell* c, double* volume, double centroid3[3], int32_t* n_faces, double* face_areas,
                    int32_t* face_neighbors) {
  int r = ready(c);
  if (r != VD_OK) return r;
  k_cell_measure<<<1, 32, 0, c->stream>>>(c->poly, c->state, c->out, c->fnb, c->farea);
  VC_CK(c, cudaGetLastError());
  CellOut h;
  r = fetch_out(c, &h);
  if (r != VD_OK) return r;
  if (volume) *volume = h.vol;
  if (centroid3) memcpy(centroid3, h.cen, sizeof(h.cen));
  if (n_faces) *n_faces = h.nfaces;
  if (face_areas && h.nfaces > 0)
    VC_CK(c, cudaMemcpyAsync(face_areas, c->farea, (size_t)h.nfaces * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (face_neighbors && h.nfaces > 0)
    VC_CK(c, cudaMemcpyAsync(face_neighbors, c->fnb, (size_t)h.nfaces * sizeof(int32_t), cudaMemcpyDeviceToHost,
                             c->stream));
  VC_CK(c, cudaStreamSynchronize(c->stream));
  return VD_OK;
}

int vd_cell_get(vd_cell* c, int32_t* n_vertices, int32_t* n_faces, int32_t* n_face_indices, double* vertices,
                uint32_t* face_counts, uint32_t* face_indices, int32_t* face_neighbors) {
  int r = ready(c);
  if (r != VD_OK) return r;
  WorkList W;
  memset(&W, 0, sizeof(W));
  W.ex_verts = c->ex_v;
  W.ex_fc = c->ex_fc;
  W.ex_fi = c->ex_fi;
  W.ex_fn = c->ex_fn;
  W.ex_sizes = c->ex_sizes;
  W.ex_cap_v = CellCfg::VCAP;
  W.ex_cap_f = CellCfg::FCAP;
  W.ex_cap_h = CellCfg::HCAP;
  k_cell_export<<<1, 32, 0, c->stream>>>(c->poly, c->state, W);
  VC_CK(c, cudaGetLastError());
  int32_t sz[4];
  VC_CK(c, cudaMemcpyAsync(sz, c->ex_sizes, sizeof(sz), cudaMemcpyDeviceToHost, c->stream));
  VC_CK(c, cudaStreamSynchronize(c->stream));
  if (n_vertices) *n_vertices = sz[0];
  if (n_faces) *n_faces = sz[1];
  if (n_face_indices) *n_face_indices = sz[2];
  if (vertices && sz[0])
    VC_CK(c, cudaMemcpyAsync(vertices, c->ex_v, 3 * (size_t)sz[0] * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (face_counts && sz[1])
    VC_CK(c, cudaMemcpyAsync(face_counts, c->ex_fc, (size_t)sz[1] * 4, cudaMemcpyDeviceToHost, c->stream));
  if (face_neighbors && sz[1])
    VC_CK(c, cudaMemcpyAsync(face_neighbors, c->ex_fn, (size_t)sz[1] * 4, cudaMemcpyDeviceToHost, c->stream));
  if (face_indices && sz[2])
    VC_CK(c, cudaMemcpyAsync(face_indices, c->ex_fi, (size_t)sz[2] * 4, cudaMemcpyDeviceToHost, c->stream));
  VC_CK(c, cudaStreamSynchronize(c->stream));
  return VD_OK;
}

}  // extern "C"
