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
  std::stable_sort(v.begin(), v.end(), [](const E& a, const E& b) { return a.o.min_d2 < b.o.min_d2; });
  out.resize(v.size());
  for (size_t i = 0; i < v.size(); ++i) out[i] = v[i].o;
}

}  // namespace vd
