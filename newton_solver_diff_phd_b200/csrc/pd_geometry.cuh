// Closest point of a triangle, shared by the mesh contact state force and the
// mesh frictional boundary.
#pragma once

#include "pd_math.cuh"

namespace pdb200 {

struct TrianglePoint {
  V3<double> point;
  V3<double> weights;
};

__device__ __forceinline__ double dot3(const V3<double>& a, const V3<double>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Closest point of triangle abc to p with its barycentric weights (Voronoi
// region tests of the reference, mesh_contact.py:34-76).
__device__ inline TrianglePoint closest_point(const V3<double>& p, const V3<double>& a, const V3<double>& b, const V3<double>& c) {
  const V3<double> ab = b - a, ac = c - a, ap = p - a;
  const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return {a, v3<double>(1.0, 0.0, 0.0)};
  const V3<double> bp = p - b;
  const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0.0 && d4 <= d3) return {b, v3<double>(0.0, 1.0, 0.0)};
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
    const double t = d1 / (d1 - d3);
    return {a + t * ab, v3<double>(1.0 - t, t, 0.0)};
  }
  const V3<double> cp = p - c;
  const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return {c, v3<double>(0.0, 0.0, 1.0)};
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
    const double t = d2 / (d2 - d6);
    return {a + t * ac, v3<double>(1.0 - t, 0.0, t)};
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
    const double t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    return {b + t * (c - b), v3<double>(0.0, 1.0 - t, t)};
  }
  const double scale = 1.0 / (va + vb + vc);
  const double v = vb * scale, w = vc * scale;
  return {a + v * ab + w * ac, v3<double>(1.0 - v - w, v, w)};
}

}  // namespace pdb200
