// vd_server.cu -- a request loop serving tessellations with continuous batching.
//
// Each request is one reference Tessellation job (bounds, grid, walls,
// generators) answered with per-cell volume, centroid and face count.  The
// server owns `slots` worker threads; each keeps one tessellation handle
// (vd_tess, with its own CUDA stream) whose device buffers stay resident and
// only grow, so a request costs no allocation once the slot has seen one of
// its size.  Admission is FIFO by HBM budget: the head of the queue starts
// as soon as a slot is free and its estimated footprint fits beside the
// requests already running.  Requests that arrive while others are on the
// GPU are admitted without waiting for them, and the slots' streams overlap
// on the device.  Small requests waiting together can be merged
// (vd_server_set_merging; off by default): a slot takes
// the run of small requests at the head of the queue and computes them as one
// batch (vd_batch: one binning pass and one persistent clip launch over a
// device work list of all their cells) instead of one calculate chain each.
// Each request's result is computed by the same kernels as a standalone
// vd_tess, so it is the same alone, in the mix and in a merged batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/voronoid_b200.h"
#include "vd_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id = 0;
  double bmin[3], bmax[3];
  int n[3];
  std::vector<vd_wall_desc> walls;
  std::vector<std::vector<double>> wall_planes;  // owned copies of polyhedron planes (points then normals)
  std::vector<double> pts;
  size_t est_bytes = 0;   // admission estimate when it runs alone
  size_t data_bytes = 0;  // its share of a merged batch's buffers
  Clock::time_point t_submit, t_start, t_done;
  bool done = false;
  bool started = false;
  bool faces = false;  // also return the neighbour-id / face-area CSR
  int status = VD_OK;
  std::string err;
  size_t ncells = 0;
  std::vector<double> vol, cen;
  std::vector<int32_t> nf;
  std::vector<int64_t> off;
  std::vector<int32_t> ids;
  std::vector<double> areas;
};

// scratch a slot may hold for cells beyond the shared-memory tiers: warps of
// large-tier polytopes and blocks of huge-tier polytopes (the persistent
// kernels run with fewer when a request has more such cells)
constexpr size_t kSlotBigWarps = 64;
constexpr size_t kSlotHugeBlocks = 8;

// device bytes a request of n generators on b bins needs: the buffers of a
// vd_tess (generators, bins, bin-ordered copy, per-cell outputs and 48 face
// slots, fallback lists), its search order, the slot's bounded large- and
// huge-tier scratch and a face pool of 2^20 slots
size_t estimate_data_bytes(size_t n, size_t bins) {
  const size_t per_cell = 24 * 3 + 32 + 4 * 6 + (8 + 24 + 4 + 4 + 1 + 8) + 48 * 12 + 3 * 4 + 8;
  return n * per_cell + bins * 16 + (1u << 20);
}

size_t estimate_bytes(size_t n, size_t bins) {
  static const size_t scratch = [] {
    vd::ClipLaunchInfo info{};
    vd::clip_fp64_info(&info);
    return kSlotBigWarps * info.big_scratch_per_warp + kSlotHugeBlocks * vd::clip_huge_scratch_per_block() +
           ((size_t)1 << 20) * 12;
  }();
  return estimate_data_bytes(n, bins) + scratch;
}

// merging: a request joins a merged batch when it asks for no face results,
// has at most max_request generators and a box and grid the standalone path
// accepts (anything else runs alone and gets the standalone path's answer)
bool mergeable(const Request& r, size_t max_request) {
  const size_t n = r.pts.size() / 3;
  if (r.faces || n == 0 || n > max_request || r.walls.size() > (size_t)vd::kMaxWalls) return false;
  for (int a = 0; a < 3; ++a) {
    if (r.n[a] <= 0 || r.n[a] > 16000) return false;
    if (!(r.bmax[a] > r.bmin[a]) || !std::isfinite(r.bmin[a]) || !std::isfinite(r.bmax[a]) ||
        !std::isfinite(r.bmax[a] - r.bmin[a]))
      return false;
  }
  return (double)r.n[0] * r.n[1] * r.n[2] <= 1.0e7;
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (double)(v.size() - 1);
  const size_t lo = (size_t)pos;
  const size_t hi = std::min(lo + 1, v.size() - 1);
  return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace

struct vd_server {
  int device = 0;
  size_t budget = 0;
  int precision = VD_PREC_FP64;
  std::string err;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
  size_t in_use = 0, peak = 0;
  int running = 0, peak_running = 0;
  bool face_results = false;
  // merging of small requests (max_members <= 1: off)
  int merge_members = 0;
  size_t merge_request = 65536, merge_group = (size_t)1 << 20;
  size_t batch_scratch = 0;
  uint64_t groups = 0, merged = 0;
  uint64_t next_id = 1;
  bool stop = false;
  std::vector<std::thread> workers;
  std::vector<vd_tess*> handles;
  std::vector<double> latencies;
  uint64_t completed = 0, cells = 0;
};

namespace {

thread_local std::string g_server_create_error;

int sfail(vd_server* s, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (s) {
    std::lock_guard<std::mutex> lock(s->mu);
    s->err = buf;
  } else {
    g_server_create_error = buf;
  }
  return code;
}

int run_request(vd_tess* t, int precision, Request& r) {
  int rc = vd_tess_reset(t, r.bmin, r.bmax, r.n[0], r.n[1], r.n[2]);
  if (rc == VD_OK) rc = vd_tess_set_precision(t, precision);
  for (size_t k = 0; k < r.walls.size() && rc == VD_OK; ++k) {
    const vd_wall_desc& w = r.walls[k];
    switch (w.kind) {
      case 0: rc = vd_tess_add_wall_plane(t, w.a, w.n, w.id); break;
      case 1: rc = vd_tess_add_wall_sphere(t, w.a, w.r, w.id); break;
      case 2: rc = vd_tess_add_wall_cylinder(t, w.a, w.n, w.r, w.id); break;
      case 3: rc = vd_tess_add_wall_cone(t, w.a, w.n, w.r, w.id); break;
      case 4: rc = vd_tess_add_wall_torus(t, w.a, w.n, w.r, w.r2, w.id); break;
      default: {
        const std::vector<double>& pl = r.wall_planes[k];
        rc = vd_tess_add_wall_polyhedron(t, pl.data(), pl.data() + 3 * w.nplanes, w.nplanes, w.id);
      }
    }
  }
  size_t kept = 0;
  if (rc == VD_OK) rc = vd_tess_set_generators(t, r.pts.data(), r.pts.size() / 3, &kept);
  if (rc == VD_OK) rc = vd_tess_calculate(t);
  if (rc == VD_OK) {
    r.ncells = kept;
    r.vol.resize(kept);
    r.cen.resize(3 * kept);
    r.nf.resize(kept);
    rc = vd_tess_get_cell_summaries(t, r.vol.data(), r.cen.data(), r.nf.data());
  }
  if (rc == VD_OK && r.faces) {
    int64_t total = 0;
    rc = vd_tess_total_faces(t, &total);
    if (rc == VD_OK) {
      r.off.resize(kept + 1);
      r.ids.resize((size_t)total);
      r.areas.resize((size_t)total);
      rc = vd_tess_get_neighbors(t, r.off.data(), r.ids.data());
    }
    if (rc == VD_OK) rc = vd_tess_get_face_areas(t, nullptr, r.areas.data());
  }
  if (rc != VD_OK) r.err = vd_last_error(t);
  return rc;
}

// the requests of a merged group computed as one batch (vd_batch_add for
// each, one commit, one calculate); false if the batch failed, and then each
// request runs alone
bool run_group(vd_batch* b, int precision, std::vector<std::shared_ptr<Request>>& g) {
  int rc = vd_batch_reset(b);
  if (rc == VD_OK) rc = vd_batch_set_precision(b, precision);
  std::vector<int> idx(g.size(), -1);
  for (size_t k = 0; k < g.size() && rc == VD_OK; ++k) {
    Request& r = *g[k];
    std::vector<vd_wall_desc> w = r.walls;
    for (size_t j = 0; j < w.size(); ++j)
      if (w[j].kind == 5 && w[j].nplanes > 0) {
        w[j].points = r.wall_planes[j].data();
        w[j].normals = r.wall_planes[j].data() + 3 * w[j].nplanes;
      }
    rc = vd_batch_add(b, r.bmin, r.bmax, r.n[0], r.n[1], r.n[2], w.data(), (int)w.size(), r.pts.data(),
                      r.pts.size() / 3, &idx[k]);
  }
  if (rc == VD_OK) rc = vd_batch_commit(b);
  if (rc == VD_OK) rc = vd_batch_calculate(b);
  for (size_t k = 0; k < g.size() && rc == VD_OK; ++k) {
    Request& r = *g[k];
    size_t n = 0;
    rc = vd_batch_count_cells(b, idx[k], &n);
    if (rc != VD_OK) break;
    r.ncells = n;
    r.vol.resize(n);
    r.cen.resize(3 * n);
    r.nf.resize(n);
    rc = vd_batch_get_summaries(b, idx[k], r.vol.data(), r.cen.data(), r.nf.data());
  }
  return rc == VD_OK;
}

void worker(vd_server* s, int slot) {
  cudaSetDevice(s->device);
  vd_tess* t = s->handles[slot];
  vd_batch* b = nullptr;  // this slot's merged batches (made for its first)
  for (;;) {
    std::vector<std::shared_ptr<Request>> g;
    size_t charge = 0;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      s->cv_work.wait(lock, [&] {
        if (s->stop) return true;
        if (s->queue.empty()) return false;
        const size_t need = s->queue.front()->est_bytes;
        return s->in_use == 0 || s->in_use + need <= s->budget;
      });
      if (s->stop) break;
      std::shared_ptr<Request> r = s->queue.front();
      s->queue.pop_front();
      g.push_back(r);
      charge = r->est_bytes;
      // the run of small requests behind it joins it, as far as the budget
      // and the group limits allow (FIFO order is kept: the run ends at the
      // first request that cannot join)
      if (s->merge_members > 1 && mergeable(*r, s->merge_request)) {
        size_t cells = r->pts.size() / 3, data = r->data_bytes;
        while ((int)g.size() < s->merge_members && !s->queue.empty()) {
          const std::shared_ptr<Request>& q = s->queue.front();
          const size_t qn = q->pts.size() / 3;
          if (!mergeable(*q, s->merge_request) || cells + qn > s->merge_group) break;
          if (s->in_use + data + q->data_bytes + s->batch_scratch > s->budget) break;
          cells += qn;
          data += q->data_bytes;
          g.push_back(q);
          s->queue.pop_front();
        }
        if (g.size() > 1) charge = data + s->batch_scratch;
      }
      s->in_use += charge;
      s->peak = std::max(s->peak, s->in_use);
      s->running += (int)g.size();
      s->peak_running = std::max(s->peak_running, s->running);
      const Clock::time_point now = Clock::now();
      for (auto& q : g) {
        q->started = true;
        q->t_start = now;
      }
    }
    // the next queued request may fit beside these
    s->cv_work.notify_all();
    std::vector<int> rcs(g.size(), VD_OK);
    bool grouped = false;
    if (g.size() > 1) {
      if (!b && vd_batch_create(&b) != VD_OK) b = nullptr;
      if (b) grouped = run_group(b, s->precision, g);
    }
    if (!grouped)
      for (size_t k = 0; k < g.size(); ++k) rcs[k] = run_request(t, s->precision, *g[k]);
    {
      std::lock_guard<std::mutex> lock(s->mu);
      s->in_use -= charge;
      s->running -= (int)g.size();
      if (grouped) {
        s->groups++;
        s->merged += g.size();
      }
      const Clock::time_point now = Clock::now();
      for (size_t k = 0; k < g.size(); ++k) {
        Request& r = *g[k];
        r.status = rcs[k];
        r.t_done = now;
        r.done = true;
        r.pts.clear();
        r.pts.shrink_to_fit();
        if (rcs[k] == VD_OK) {
          s->latencies.push_back(std::chrono::duration<double>(r.t_done - r.t_submit).count());
          s->completed++;
          s->cells += r.ncells;
        }
      }
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
  if (b) vd_batch_destroy(b);
}

// the request's clock starts at t0 (before parsing, for a text request)
int submit_points(vd_server* s, const double bmin[3], const double bmax[3], int nx, int ny, int nz,
                  const vd_wall_desc* walls, int nwalls, std::vector<double>&& pts, Clock::time_point t0,
                  uint64_t* ticket) {
  const size_t n = pts.size() / 3;
  if (nx <= 0 || ny <= 0 || nz <= 0) return sfail(s, VD_EINVAL, "grid resolution must be positive");
  for (int k = 0; k < nwalls; ++k) {
    const vd_wall_desc& w = walls[k];
    if (w.id > VD_WALL_ID_MAX || w.kind < 0 || w.kind > 5 ||
        (w.kind == 5 && (w.nplanes < 0 || (w.nplanes > 0 && (!w.points || !w.normals)))))
      return sfail(s, VD_EINVAL, "bad wall %d", k);
  }
  auto r = std::make_shared<Request>();
  for (int a = 0; a < 3; ++a) {
    r->bmin[a] = bmin[a];
    r->bmax[a] = bmax[a];
  }
  r->n[0] = nx;
  r->n[1] = ny;
  r->n[2] = nz;
  r->walls.assign(walls, walls + nwalls);
  r->wall_planes.resize(nwalls);
  for (int k = 0; k < nwalls; ++k) {
    vd_wall_desc& w = r->walls[k];
    if (w.kind == 5 && w.nplanes > 0) {
      r->wall_planes[k].assign(w.points, w.points + 3 * w.nplanes);
      r->wall_planes[k].insert(r->wall_planes[k].end(), w.normals, w.normals + 3 * w.nplanes);
    }
    w.points = w.normals = nullptr;  // the request keeps its own copy
  }
  r->pts = std::move(pts);
  r->faces = s->face_results;
  r->est_bytes = estimate_bytes(n, (size_t)nx * ny * nz);
  r->data_bytes = estimate_data_bytes(n, (size_t)nx * ny * nz);
  if (r->est_bytes > s->budget) return sfail(s, VD_ENOMEM, "request needs %zu bytes, budget %zu", r->est_bytes, s->budget);
  {
    std::lock_guard<std::mutex> lock(s->mu);
    r->id = s->next_id++;
    r->t_submit = t0;
    s->live[r->id] = r;
    s->queue.push_back(r);
    *ticket = r->id;
  }
  s->cv_work.notify_all();
  return VD_OK;
}

}  // namespace

extern "C" {

const char* vd_server_last_error(const vd_server* s) {
  return s ? s->err.c_str() : g_server_create_error.c_str();
}

int vd_server_create(int slots, size_t hbm_budget_bytes, int precision, vd_server** out) {
  if (!out || slots <= 0 || slots > 256) return sfail(nullptr, VD_EINVAL, "slots must be in [1, 256]");
  if (precision != VD_PREC_FP64 && precision != VD_PREC_MIXED) return sfail(nullptr, VD_EINVAL, "unknown precision");
  *out = nullptr;
  vd_server* s = new vd_server();
  if (cudaGetDevice(&s->device) != cudaSuccess) {
    delete s;
    return sfail(nullptr, VD_ECUDA, "no CUDA device");
  }
  s->budget = hbm_budget_bytes;
  s->precision = precision;
  {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    s->batch_scratch = vd::batch_scratch_bytes(sms);
  }
  const double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  for (int k = 0; k < slots; ++k) {
    vd_tess* t = nullptr;
    const int rc = vd_tess_create(lo, hi, 1, 1, 1, &t);
    if (rc != VD_OK) {
      const std::string m = vd_last_error(nullptr);
      for (vd_tess* h : s->handles) vd_tess_destroy(h);
      delete s;
      return sfail(nullptr, rc, "slot setup: %s", m.c_str());
    }
    vd::set_scratch_caps(t, kSlotBigWarps, kSlotHugeBlocks);
    s->handles.push_back(t);
  }
  // Reserve the budget in the library's memory pool up front (as much of it
  // as the device has free): a request that grows its slot's buffers is then
  // served from the pool instead of the driver.  Best effort.
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
    void* st = nullptr;
    vd_tess_stream(s->handles[0], &st);
    for (size_t want = std::min(hbm_budget_bytes, free_b / 10 * 9); want >= ((size_t)1 << 28); want /= 2)
      if (vd::reserve_pool(want, (cudaStream_t)st) == cudaSuccess) break;
    cudaGetLastError();
  }
  for (int k = 0; k < slots; ++k) s->workers.emplace_back(worker, s, k);
  *out = s;
  return VD_OK;
}

int vd_server_destroy(vd_server* s) {
  if (!s) return VD_OK;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& w : s->workers) w.join();
  for (vd_tess* t : s->handles) vd_tess_destroy(t);
  delete s;
  return VD_OK;
}


int vd_server_submit(vd_server* s, const double bmin[3], const double bmax[3], int nx, int ny, int nz,
                     const vd_wall_desc* walls, int nwalls, const double* xyz, size_t n, uint64_t* ticket) {
  if (!s || !bmin || !bmax || !ticket || (!xyz && n) || (nwalls > 0 && !walls) || nwalls < 0)
    return VD_EINVAL;
  const Clock::time_point t0 = Clock::now();
  return submit_points(s, bmin, bmax, nx, ny, nz, walls, nwalls, std::vector<double>(xyz, xyz + 3 * n), t0,
                       ticket);
}

// a request whose generators arrive in the text format of
// Tessellation::read_generators (tessellation.rs:153-171); parsed here, on the
// submitting thread, inside the request's latency
int vd_server_submit_text(vd_server* s, const double bmin[3], const double bmax[3], int nx, int ny, int nz,
                          const vd_wall_desc* walls, int nwalls, const char* text, size_t len, uint64_t* ticket) {
  if (!s || !bmin || !bmax || !ticket || (!text && len) || (nwalls > 0 && !walls) || nwalls < 0)
    return VD_EINVAL;
  const Clock::time_point t0 = Clock::now();
  std::vector<double> pts;
  std::string err;
  if (!vd::parse_generators(text, len, &pts, &err)) return sfail(s, VD_EINVAL, "%s", err.c_str());
  return submit_points(s, bmin, bmax, nx, ny, nz, walls, nwalls, std::move(pts), t0, ticket);
}

int vd_server_wait(vd_server* s, uint64_t ticket, size_t* n_cells, double* latency_s) {
  if (!s) return VD_EINVAL;
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->live.find(ticket);
  if (it == s->live.end()) {
    s->err = "unknown ticket";
    return VD_EINVAL;
  }
  std::shared_ptr<Request> r = it->second;
  s->cv_done.wait(lock, [&] { return r->done; });
  if (n_cells) *n_cells = r->ncells;
  if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  if (r->status != VD_OK) s->err = r->err;
  return r->status;
}

int vd_server_take(vd_server* s, uint64_t ticket, double* volume, double* centroid3, int32_t* n_faces) {
  if (!s) return VD_EINVAL;
  std::shared_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->live.find(ticket);
    if (it == s->live.end()) {
      s->err = "unknown ticket";
      return VD_EINVAL;
    }
    r = it->second;
    s->cv_done.wait(lock, [&] { return r->done; });
    s->live.erase(it);
  }
  if (r->status != VD_OK) return r->status;
  if (volume) memcpy(volume, r->vol.data(), r->ncells * sizeof(double));
  if (centroid3) memcpy(centroid3, r->cen.data(), 3 * r->ncells * sizeof(double));
  if (n_faces) memcpy(n_faces, r->nf.data(), r->ncells * sizeof(int32_t));
  return VD_OK;
}

int vd_server_take_faces(vd_server* s, uint64_t ticket, double* volume, double* centroid3, int32_t* n_faces,
                         int64_t* offsets, int32_t* ids, double* areas) {
  if (!s) return VD_EINVAL;
  std::shared_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->live.find(ticket);
    if (it == s->live.end()) {
      s->err = "unknown ticket";
      return VD_EINVAL;
    }
    r = it->second;
    s->cv_done.wait(lock, [&] { return r->done; });
    if (r->status == VD_OK && !r->faces && (offsets || ids || areas)) {
      s->err = "the request was submitted without face results (vd_server_set_face_results)";
      return VD_ESTATE;
    }
    s->live.erase(it);
  }
  if (r->status != VD_OK) return r->status;
  if (volume) memcpy(volume, r->vol.data(), r->ncells * sizeof(double));
  if (centroid3) memcpy(centroid3, r->cen.data(), 3 * r->ncells * sizeof(double));
  if (n_faces) memcpy(n_faces, r->nf.data(), r->ncells * sizeof(int32_t));
  if (r->faces) {
    if (offsets) memcpy(offsets, r->off.data(), r->off.size() * sizeof(int64_t));
    if (ids) memcpy(ids, r->ids.data(), r->ids.size() * sizeof(int32_t));
    if (areas) memcpy(areas, r->areas.data(), r->areas.size() * sizeof(double));
  }
  return VD_OK;
}

int vd_server_total_faces(vd_server* s, uint64_t ticket, int64_t* total) {
  if (!s || !total) return VD_EINVAL;
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->live.find(ticket);
  if (it == s->live.end()) {
    s->err = "unknown ticket";
    return VD_EINVAL;
  }
  std::shared_ptr<Request> r = it->second;
  s->cv_done.wait(lock, [&] { return r->done; });
  *total = (int64_t)r->ids.size();
  if (r->status != VD_OK) s->err = r->err;
  return r->status;
}

int vd_server_set_face_results(vd_server* s, int on) {
  if (!s) return VD_EINVAL;
  std::lock_guard<std::mutex> lock(s->mu);
  s->face_results = on != 0;
  return VD_OK;
}

int vd_server_cancel(vd_server* s, uint64_t ticket) {
  if (!s) return VD_EINVAL;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->live.find(ticket);
    if (it == s->live.end()) {
      s->err = "unknown ticket";
      return VD_EINVAL;
    }
    std::shared_ptr<Request> r = it->second;
    if (r->started || r->done) {
      s->err = "the request has already started";
      return VD_ESTATE;
    }
    s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
    r->status = VD_ECANCELED;
    r->err = "cancelled";
    r->t_done = Clock::now();
    r->done = true;
    r->pts.clear();
    r->pts.shrink_to_fit();
  }
  s->cv_done.notify_all();
  s->cv_work.notify_all();  // the next request may fit now
  return VD_OK;
}

int vd_server_set_merging(vd_server* s, int max_members, size_t max_request, size_t max_group) {
  if (!s || max_members < 0) return VD_EINVAL;
  std::lock_guard<std::mutex> lock(s->mu);
  s->merge_members = max_members;
  if (max_request) s->merge_request = max_request;
  if (max_group) s->merge_group = max_group;
  return VD_OK;
}

int vd_server_merge_stats(vd_server* s, uint64_t* groups, uint64_t* merged_requests) {
  if (!s) return VD_EINVAL;
  std::lock_guard<std::mutex> lock(s->mu);
  if (groups) *groups = s->groups;
  if (merged_requests) *merged_requests = s->merged;
  return VD_OK;
}

int vd_server_concurrency(vd_server* s, int* running, int* peak_running) {
  if (!s) return VD_EINVAL;
  std::lock_guard<std::mutex> lock(s->mu);
  if (running) *running = s->running;
  if (peak_running) *peak_running = s->peak_running;
  return VD_OK;
}

int vd_server_stats(vd_server* s, uint64_t* completed, uint64_t* cells, double* p50_s, double* p99_s,
                    size_t* peak_bytes) {
  if (!s) return VD_EINVAL;
  std::lock_guard<std::mutex> lock(s->mu);
  if (completed) *completed = s->completed;
  if (cells) *cells = s->cells;
  if (p50_s) *p50_s = percentile(s->latencies, 0.50);
  if (p99_s) *p99_s = percentile(s->latencies, 0.99);
  if (peak_bytes) *peak_bytes = s->peak;
  return VD_OK;
}

int vd_server_reset_stats(vd_server* s) {
  if (!s) return VD_EINVAL;
  std::lock_guard<std::mutex> lock(s->mu);
  s->latencies.clear();
  s->completed = 0;
  s->cells = 0;
  s->peak = s->in_use;
  s->peak_running = s->running;
  s->groups = 0;
  s->merged = 0;
  return VD_OK;
}

}  // extern "C"
