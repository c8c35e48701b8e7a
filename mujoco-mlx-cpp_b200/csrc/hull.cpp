#include "hull.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <set>
#include <utility>

namespace mjb {
namespace {

struct V3 {
  double x, y, z;
};
V3 at(const std::vector<double>& p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
double norm(V3 a) { return std::sqrt(dot(a, a)); }

}  // namespace

ConvexHull convex_hull(const std::vector<double>& pts) {
  ConvexHull h;
  h.points = pts;
  int n = (int)pts.size() / 3;
  if (n < 4) return h;
  double scale = 0;
  for (int i = 0; i < n; i++) scale = std::max(scale, norm(at(pts, i)));
  double eps = 1e-10 * std::max(scale, 1e-6);
  // initial tetrahedron: extreme x pair, farthest from line, farthest from plane
  int i0 = 0, i1 = 0;
  for (int i = 1; i < n; i++) {
    if (pts[3 * i] < pts[3 * i0]) i0 = i;
    if (pts[3 * i] > pts[3 * i1]) i1 = i;
  }
  if (i0 == i1) {
    for (int i = 0; i < n; i++)
      if (norm(sub(at(pts, i), at(pts, i0))) > eps) { i1 = i; break; }
    if (i0 == i1) return h;
  }
  V3 a = at(pts, i0), b = at(pts, i1);
  int i2 = -1;
  double best = eps;
  for (int i = 0; i < n; i++) {
    double d = norm(cross(sub(at(pts, i), a), sub(b, a)));
    if (d > best) { best = d; i2 = i; }
  }
  if (i2 < 0) return h;
  V3 c = at(pts, i2);
  V3 nrm = cross(sub(b, a), sub(c, a));
  int i3 = -1;
  best = eps * norm(nrm);
  for (int i = 0; i < n; i++) {
    double d = std::fabs(dot(nrm, sub(at(pts, i), a)));
    if (d > best) { best = d; i3 = i; }
  }
  if (i3 < 0) return h;
  std::vector<std::array<int, 3>> faces;
  auto add_face = [&](int p, int q, int r, V3 inside) {
    V3 fn = cross(sub(at(pts, q), at(pts, p)), sub(at(pts, r), at(pts, p)));
    if (dot(fn, sub(inside, at(pts, p))) > 0) std::swap(q, r);
    faces.push_back({p, q, r});
  };
  V3 cen = {(a.x + b.x + c.x + pts[3 * i3]) / 4, (a.y + b.y + c.y + pts[3 * i3 + 1]) / 4, (a.z + b.z + c.z + pts[3 * i3 + 2]) / 4};
  add_face(i0, i1, i2, cen);
  add_face(i0, i1, i3, cen);
  add_face(i0, i2, i3, cen);
  add_face(i1, i2, i3, cen);
  std::set<int> used = {i0, i1, i2, i3};
  for (int i = 0; i < n; i++) {
    if (used.count(i)) continue;
    V3 p = at(pts, i);
    std::vector<char> visible(faces.size(), 0);
    bool any = false;
    for (size_t f = 0; f < faces.size(); f++) {
      V3 fa = at(pts, faces[f][0]);
      V3 fn = cross(sub(at(pts, faces[f][1]), fa), sub(at(pts, faces[f][2]), fa));
      double l = norm(fn);
      if (l < 1e-300) continue;
      if (dot(fn, sub(p, fa)) / l > eps) { visible[f] = 1; any = true; }
    }
    if (!any) continue;
    // horizon: directed edges of visible faces whose reverse is not on a visible face
    std::map<std::pair<int, int>, int> edges;
    for (size_t f = 0; f < faces.size(); f++)
      if (visible[f])
        for (int k = 0; k < 3; k++) edges[{faces[f][k], faces[f][(k + 1) % 3]}]++;
    std::vector<std::array<int, 3>> kept;
    for (size_t f = 0; f < faces.size(); f++)
      if (!visible[f]) kept.push_back(faces[f]);
    for (auto& e : edges)
      if (!edges.count({e.first.second, e.first.first})) kept.push_back({e.first.first, e.first.second, i});
    faces.swap(kept);
  }
  std::set<int> vids;
  for (auto& f : faces)
    for (int k = 0; k < 3; k++) vids.insert(f[k]);
  h.vertex_ids.assign(vids.begin(), vids.end());
  h.faces = faces;
  return h;
}

void hull_mass_properties(const ConvexHull& h, double& volume, double com[3], double I[9]) {
  const auto& p = h.points;
  double V = 0, c[3] = {0, 0, 0}, C[9] = {0};
  for (auto& f : h.faces) {
    V3 a = at(p, f[0]), b = at(p, f[1]), d = at(p, f[2]);
    double v = dot(a, cross(b, d)) / 6;  // signed volume of tetra (0, a, b, d)
    V += v;
    double s[3] = {a.x + b.x + d.x, a.y + b.y + d.y, a.z + b.z + d.z};
    for (int k = 0; k < 3; k++) c[k] += v * s[k] / 4;
    double va[3] = {a.x, a.y, a.z}, vb[3] = {b.x, b.y, b.z}, vd[3] = {d.x, d.y, d.z};
    for (int r = 0; r < 3; r++)
      for (int q = 0; q < 3; q++)
        C[r * 3 + q] += v / 20 * (va[r] * va[q] + vb[r] * vb[q] + vd[r] * vd[q] + s[r] * s[q]);
  }
  volume = V;
  for (int k = 0; k < 3; k++) com[k] = V > 0 ? c[k] / V : 0;
  double tr = C[0] + C[4] + C[8];
  for (int r = 0; r < 3; r++)
    for (int q = 0; q < 3; q++) I[r * 3 + q] = (r == q ? tr : 0) - C[r * 3 + q];
  double c2 = com[0] * com[0] + com[1] * com[1] + com[2] * com[2];
  for (int r = 0; r < 3; r++)
    for (int q = 0; q < 3; q++) I[r * 3 + q] -= V * ((r == q ? c2 : 0) - com[r] * com[q]);
}

}  // namespace mjb
