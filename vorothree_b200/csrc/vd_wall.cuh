// vd_wall.cuh -- the plane a wall emits for one generator (WallGeometry::cut),
// shared by the clip kernels and the host-side wall queries (vd_wall_cut).
// Host code is built with -ffp-contract=off and the kernels with -fmad=false,
// and sqrt and division are correctly rounded on both, so the two agree bit
// for bit.
#pragma once
#include <cmath>

#include "vd_common.cuh"

namespace vd {

// WallGeometry::cut (wall_3d.rs:38-42, 80-100, 145-173, 216-261, 311-364) for
// the walls that emit one plane per generator: (p, n) with n pointing out of
// the valid region.  Returns false when the wall emits no plane.
// Convex-polyhedron walls emit their fixed planes (compute_cell).
__host__ __device__ __forceinline__ bool wall_plane(const Wall& w, double gx, double gy, double gz, double* p,
                                                    double* n) {
  if (w.kind == kWallPlane) {
    p[0] = w.a[0];
    p[1] = w.a[1];
    p[2] = w.a[2];
    n[0] = -w.n[0];
    n[1] = -w.n[1];
    n[2] = -w.n[2];
    return true;
  }
  const double dx = gx - w.a[0], dy = gy - w.a[1], dz = gz - w.a[2];
  if (w.kind == kWallSphere) {
    const double dist = sqrt(dx * dx + dy * dy + dz * dz);
    if (dist == 0.0) return false;
    const double scale = w.r / dist;
    p[0] = w.a[0] + dx * scale;
    p[1] = w.a[1] + dy * scale;
    p[2] = w.a[2] + dz * scale;
    n[0] = dx / dist;
    n[1] = dy / dist;
    n[2] = dz / dist;
    return true;
  }
  const double dot = dx * w.n[0] + dy * w.n[1] + dz * w.n[2];
  const double px = dx - dot * w.n[0], py = dy - dot * w.n[1], pz = dz - dot * w.n[2];
  const double rp = sqrt(px * px + py * py + pz * pz);
  if (w.kind == kWallCylinder) {
    if (rp == 0.0) return false;
    const double scale = w.r / rp;
    p[0] = w.a[0] + dot * w.n[0] + px * scale;
    p[1] = w.a[1] + dot * w.n[1] + py * scale;
    p[2] = w.a[2] + dot * w.n[2] + pz * scale;
    n[0] = px / rp;
    n[1] = py / rp;
    n[2] = pz / rp;
    return true;
  }
  if (w.kind == kWallCone) {
    // dot is the height h along the axis, rp the distance r from it
    if (rp == 0.0) return false;
    const double ux = px / rp, uy = py / rp, uz = pz / rp;
    const double dist = rp * w.ca - dot * w.sa;
    const double pr = rp - dist * w.ca;
    const double ph = dot + dist * w.sa;
    if (ph < 0.0) {
      const double dt = sqrt(dx * dx + dy * dy + dz * dz);
      if (dt == 0.0) return false;
      p[0] = w.a[0];
      p[1] = w.a[1];
      p[2] = w.a[2];
      n[0] = dx / dt;
      n[1] = dy / dt;
      n[2] = dz / dt;
      return true;
    }
    p[0] = w.a[0] + ph * w.n[0] + pr * ux;
    p[1] = w.a[1] + ph * w.n[1] + pr * uy;
    p[2] = w.a[2] + ph * w.n[2] + pr * uz;
    n[0] = w.ca * ux - w.sa * w.n[0];
    n[1] = w.ca * uy - w.sa * w.n[1];
    n[2] = w.ca * uz - w.sa * w.n[2];
    return true;
  }
  // torus: the nearest point of the major circle, then the tube's tangent plane
  double ux, uy, uz;
  if (rp < 1e-9) {
    double tx = 1.0, ty = 0.0;
    const double tz = 0.0;
    if (fabs(w.n[0]) > 0.9) {
      tx = 0.0;
      ty = 1.0;
    }
    const double td = tx * w.n[0] + ty * w.n[1] + tz * w.n[2];
    const double ax = tx - td * w.n[0], ay = ty - td * w.n[1], az = tz - td * w.n[2];
    const double len = sqrt(ax * ax + ay * ay + az * az);
    if (len == 0.0) return false;
    ux = ax / len;
    uy = ay / len;
    uz = az / len;
  } else {
    ux = px / rp;
    uy = py / rp;
    uz = pz / rp;
  }
  const double cx = w.a[0] + ux * w.r, cy = w.a[1] + uy * w.r, cz = w.a[2] + uz * w.r;
  const double vx = gx - cx, vy = gy - cy, vz = gz - cz;
  const double dc = sqrt(vx * vx + vy * vy + vz * vz);
  if (dc == 0.0) return false;
  n[0] = vx / dc;
  n[1] = vy / dc;
  n[2] = vz / dc;
  p[0] = cx + n[0] * w.r2;
  p[1] = cy + n[1] * w.r2;
  p[2] = cz + n[2] * w.r2;
  return true;
}

}  // namespace vd
