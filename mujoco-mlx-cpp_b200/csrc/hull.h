// Convex hull of a point cloud (incremental algorithm, O(n^2), meant for the
// few-dozen-vertex meshes of convex collision geoms) and the mass properties
// of the resulting closed polyhedron at unit density.
#pragma once
#include <array>
#include <vector>

namespace mjb {

struct ConvexHull {
  std::vector<double> points;               // copy of the input points (xyz triples)
  std::vector<int> vertex_ids;              // input indices of hull vertices, ascending
  std::vector<std::array<int, 3>> faces;    // outward-oriented triangles (input indices)
};

// points: xyz triples.  Returns an empty face list when all points are
// (nearly) coplanar.
ConvexHull convex_hull(const std::vector<double>& points);

// Volume, centre of mass and inertia tensor about the centre of mass (row
// major 3x3), unit density.
void hull_mass_properties(const ConvexHull& h, double& volume, double com[3], double I[9]);

}  // namespace mjb
