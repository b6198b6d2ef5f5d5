// vd_order.h -- host-side construction of the shell search order.
#pragma once
#include <algorithm>
#include <cstdint>
#include <limits>
#include <vector>

#include "vd_common.cuh"

namespace vd {

// Algorithm3DGrid::new's search order (algo_3d_grid.rs:56-76): every offset
// of [-n,n]^3 (z outer, x inner) with its min_d2, sorted by min_d2.  Ties
// keep the enumeration order (a stable sort; the reference's unstable sort has
// no reproducible tie order).  With k < n the table holds exactly the offsets
// with min_d2 < bound, where bound = min over truncated axes of (k*cs)^2 is a
// lower bound of min_d2 for every offset left out.
inline void build_order(const Grid& g, int k, std::vector<Offset>& out, bool& complete, double& bound) {
  int r[3];
  complete = true;
  bound = std::numeric_limits<double>::infinity();
  for (int a = 0; a < 3; ++a) {
    r[a] = std::min(k, g.n[a]);
    if (r[a] < g.n[a]) {
      complete = false;
      const double m = (double)k * g.cs[a];
      bound = std::min(bound, m * m);
    }
  }
  struct E {
    Offset o;
    uint32_t lin;
  };
  std::vector<E> v;
  v.reserve((size_t)(2 * r[0] + 1) * (2 * r[1] + 1) * (2 * r[2] + 1));
  uint32_t lin = 0;
  for (int z = -r[2]; z <= r[2]; ++z)
    for (int y = -r[1]; y <= r[1]; ++y)
      for (int x = -r[0]; x <= r[0]; ++x) {
        const double mx = x > 0 ? (double)(x - 1) * g.cs[0] : (x < 0 ? (double)(-x - 1) * g.cs[0] : 0.0);
        const double my = y > 0 ? (double)(y - 1) * g.cs[1] : (y < 0 ? (double)(-y - 1) * g.cs[1] : 0.0);
        const double mz = z > 0 ? (double)(z - 1) * g.cs[2] : (z < 0 ? (double)(-z - 1) * g.cs[2] : 0.0);
        const double d2 = mx * mx + my * my + mz * mz;
        if (complete || d2 < bound) {
          E e;
          e.o.dx = (int16_t)x;
          e.o.dy = (int16_t)y;
          e.o.dz = (int16_t)z;
          e.o.pad = 0;
          e.o.min_d2 = d2;
          e.lin = lin;
          v.push_back(e);
        }
        ++lin;
      }
  const auto by_d2 = [](const E& a, const E& b) { return a.o.min_d2 < b.o.min_d2; };
  const int rm = std::max(r[0], std::max(r[1], r[2]));
  const uint64_t kmax = 3ull * (uint64_t)rm * (uint64_t)rm;
  if (g.cs[0] == g.cs[1] && g.cs[1] == g.cs[2] && kmax < (1ull << 24)) {
    // Cubic bins: min_d2 = cs^2 * K up to rounding, K = mx^2 + my^2 + mz^2 an
    // integer.  Two different K never swap order under rounding (the relative
    // error is ~1e-15, the relative gap between integers below 2^24 is
    // >= 6e-8), so a stable counting sort by K followed by a stable sort of
    // each bucket by the value gives exactly the stable sort by value, in
    // linear time instead of n log n.
    const auto key = [](const Offset& o) {
      const uint64_t mx = o.dx > 0 ? o.dx - 1 : (o.dx < 0 ? -o.dx - 1 : 0);
      const uint64_t my = o.dy > 0 ? o.dy - 1 : (o.dy < 0 ? -o.dy - 1 : 0);
      const uint64_t mz = o.dz > 0 ? o.dz - 1 : (o.dz < 0 ? -o.dz - 1 : 0);
      return mx * mx + my * my + mz * mz;
    };
    std::vector<uint32_t> start(kmax + 2, 0);
    for (const E& e : v) ++start[key(e.o) + 1];
    for (uint64_t q = 0; q <= kmax; ++q) start[q + 1] += start[q];
    std::vector<E> w(v.size());
    std::vector<uint32_t> pos(start.begin(), start.end() - 1);
    for (const E& e : v) w[pos[key(e.o)]++] = e;
    for (uint64_t q = 0; q <= kmax; ++q)
      if (start[q + 1] - start[q] > 1) std::stable_sort(w.begin() + start[q], w.begin() + start[q + 1], by_d2);
    v.swap(w);
  } else {
    std::stable_sort(v.begin(), v.end(), by_d2);
  }
  out.resize(v.size());
  for (size_t i = 0; i < v.size(); ++i) out[i] = v[i].o;
}

}  // namespace vd
