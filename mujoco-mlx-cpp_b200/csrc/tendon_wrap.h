// Spatial tendon wrapping geometry (MuJoCo's sphere / cylinder wrapping
// semantics, reference: tendon.hpp tw_wrap_circle / tw_wrap), shared by the
// model compiler (rest length and invweight at qpos0, host) and the step
// kernel (device).  Written from the geometry of tangent lines to a circle:
//
// * 2D: a path from p0 to p1 (both outside a circle of radius r at the
//   origin) wraps when the straight segment enters the circle, or when a
//   side point is given and the segment passes on the other side.  It then
//   runs along the tangent from p0, around the arc, and along the tangent to
//   p1; of the two senses (counter-clockwise: p0's tangent point rotated
//   +acos(r/|p0|), p1's rotated -acos(r/|p1|); clockwise the mirror) it takes
//   the one whose arc midpoint lies towards the side point, or without one
//   the one with the closer tangent points.  A sense whose two tangent
//   segments cross is invalid.
// * Sphere: the 2D problem in the plane through the centre and both path
//   points.  Cylinder: the 2D problem in the plane normal to the axis; the
//   axial coordinate of the tangent points advances in proportion to the 2D
//   path length (a helix when unrolled).
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define MJB_HD __host__ __device__ __forceinline__
#else
#define MJB_HD inline
#endif

namespace mjbwrap {

template <class T>
MJB_HD T dot3(const T* a, const T* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// segments p1-p2 and p3-p4 cross (2D)
template <class T>
MJB_HD bool crossing(const T* p1, const T* p2, const T* p3, const T* p4) {
  const T det = (p4[1] - p3[1]) * (p2[0] - p1[0]) - (p4[0] - p3[0]) * (p2[1] - p1[1]);
  if (fabs((double)det) < 1e-15) return false;
  const T a = ((p4[0] - p3[0]) * (p1[1] - p3[1]) - (p4[1] - p3[1]) * (p1[0] - p3[0])) / det;
  const T b = ((p2[0] - p1[0]) * (p1[1] - p3[1]) - (p2[1] - p1[1]) * (p1[0] - p3[0])) / det;
  return a >= 0 && a <= 1 && b >= 0 && b <= 1;
}

// tangent point of p (|p| = d > r) rotated by sgn * acos(r / d) from p's direction
template <class T>
MJB_HD void tangent(const T* p, T r, T sgn, T* t) {
  const T d = sqrt(p[0] * p[0] + p[1] * p[1]);
  const T c = r / d, s = sqrt(T(1) - c * c) * sgn;
  const T u[2] = {p[0] / d, p[1] / d};
  t[0] = r * (c * u[0] - s * u[1]);
  t[1] = r * (c * u[1] + s * u[0]);
}

// Returns the arc length when the path wraps (tangent points t0, t1), -1
// when the straight segment is the path.  side may be null.
template <class T>
MJB_HD T circle(const T* p0, const T* p1, T r, const T* side, T* t0, T* t1) {
  const T r2 = r * r;
  const T l0 = p0[0] * p0[0] + p0[1] * p0[1], l1 = p1[0] * p1[0] + p1[1] * p1[1];
  if (r <= T(0) || l0 <= r2 || l1 <= r2) return T(-1);
  const T e[2] = {p1[0] - p0[0], p1[1] - p0[1]};
  const T ee = e[0] * e[0] + e[1] * e[1];
  T a = ee > T(0) ? -(p0[0] * e[0] + p0[1] * e[1]) / ee : T(0);
  a = a < T(0) ? T(0) : (a > T(1) ? T(1) : a);
  const T q[2] = {p0[0] + a * e[0], p0[1] + a * e[1]};
  if (q[0] * q[0] + q[1] * q[1] > r2 && (!side || side[0] * q[0] + side[1] * q[1] >= T(0))) return T(-1);
  T best_g = T(0), ta[2][2], tb[2][2], arc[2];
  int best = -1;
  for (int k = 0; k < 2; k++) {
    const T sg = k == 0 ? T(1) : T(-1);   // 0: counter-clockwise around the circle, 1: clockwise
    tangent(p0, r, sg, ta[k]);
    tangent(p1, r, -sg, tb[k]);
    // arc from ta to tb in the sense sg
    T ang = atan2(ta[k][0] * tb[k][1] - ta[k][1] * tb[k][0], ta[k][0] * tb[k][0] + ta[k][1] * tb[k][1]) * sg;
    if (ang < T(0)) ang += T(6.283185307179586);
    arc[k] = r * ang;
    T g;
    if (side) {
      T mid[2] = {ta[k][0] + tb[k][0], ta[k][1] + tb[k][1]};
      const T lm = sqrt(mid[0] * mid[0] + mid[1] * mid[1]);
      if (lm > T(1e-12)) { mid[0] /= lm; mid[1] /= lm; }
      else { mid[0] = T(1); mid[1] = T(0); }
      g = mid[0] * side[0] + mid[1] * side[1];
    } else {
      const T dx = ta[k][0] - tb[k][0], dy = ta[k][1] - tb[k][1];
      g = -(dx * dx + dy * dy);
    }
    if (crossing(p0, ta[k], p1, tb[k])) g = T(-1e4);
    if (best < 0 || g > best_g) { best = k; best_g = g; }
  }
  if (crossing(p0, ta[best], p1, tb[best])) return T(-1);
  t0[0] = ta[best][0]; t0[1] = ta[best][1];
  t1[0] = tb[best][0]; t1[1] = tb[best][1];
  return arc[best];
}

// Path from s0 to s1 around a sphere (type 2) or cylinder (type 5) geom with
// centre c, rotation R (row-major, columns = geom axes) and radius r.
// side (world point) may be null.  Returns the path length; wrapped tells
// whether it left the straight line, with tangent points t0, t1 (world).
template <class T>
MJB_HD T geom(int type, const T* c, const T* R, T r, const T* s0, const T* s1, const T* side, T* t0, T* t1, bool& wrapped) {
  wrapped = false;
  const T d0[3] = {s0[0] - c[0], s0[1] - c[1], s0[2] - c[2]}, d1[3] = {s1[0] - c[0], s1[1] - c[1], s1[2] - c[2]};
  const T straight = sqrt((s1[0] - s0[0]) * (s1[0] - s0[0]) + (s1[1] - s0[1]) * (s1[1] - s0[1]) + (s1[2] - s0[2]) * (s1[2] - s0[2]));
  T e1[3], e2[3];
  T z0 = 0, z1 = 0;
  if (type == 5) {
    for (int k = 0; k < 3; k++) { e1[k] = R[3 * k]; e2[k] = R[3 * k + 1]; }
    const T ax[3] = {R[2], R[5], R[8]};
    z0 = dot3(d0, ax);
    z1 = dot3(d1, ax);
  } else {
    // plane through the centre and both points; basis e1 along s0
    const T l0 = sqrt(dot3(d0, d0));
    if (l0 < T(1e-12)) return straight;
    for (int k = 0; k < 3; k++) e1[k] = d0[k] / l0;
    const T p = dot3(d1, e1);
    T w[3] = {d1[0] - p * e1[0], d1[1] - p * e1[1], d1[2] - p * e1[2]};
    T lw = sqrt(dot3(w, w));
    if (lw < T(1e-12) * (T(1) + sqrt(dot3(d1, d1)))) {
      // collinear with the centre: use the side point, else any normal
      if (side) {
        const T ds[3] = {side[0] - c[0], side[1] - c[1], side[2] - c[2]};
        const T ps = dot3(ds, e1);
        for (int k = 0; k < 3; k++) w[k] = ds[k] - ps * e1[k];
        lw = sqrt(dot3(w, w));
      }
      if (lw < T(1e-12)) {
        const T a[3] = {fabs((double)e1[0]) < 0.6 ? T(1) : T(0), fabs((double)e1[0]) < 0.6 ? T(0) : T(1), T(0)};
        const T pa = dot3(a, e1);
        for (int k = 0; k < 3; k++) w[k] = a[k] - pa * e1[k];
        lw = sqrt(dot3(w, w));
      }
    }
    for (int k = 0; k < 3; k++) e2[k] = w[k] / lw;
  }
  const T p0[2] = {dot3(d0, e1), dot3(d0, e2)}, p1[2] = {dot3(d1, e1), dot3(d1, e2)};
  T sd[2];
  const T* sdp = nullptr;
  if (side) {
    const T ds[3] = {side[0] - c[0], side[1] - c[1], side[2] - c[2]};
    sd[0] = dot3(ds, e1);
    sd[1] = dot3(ds, e2);
    sdp = sd;
  }
  T a2[2], b2[2];
  const T arc = circle(p0, p1, r, sdp, a2, b2);
  if (arc < T(0)) return straight;
  wrapped = true;
  const T la = sqrt((a2[0] - p0[0]) * (a2[0] - p0[0]) + (a2[1] - p0[1]) * (a2[1] - p0[1]));
  const T lb = sqrt((p1[0] - b2[0]) * (p1[0] - b2[0]) + (p1[1] - b2[1]) * (p1[1] - b2[1]));
  const T L2 = la + arc + lb;
  T za = 0, zb = 0;
  T len = L2;
  if (type == 5) {
    const T dz = z1 - z0;
    za = z0 + (L2 > T(0) ? dz * la / L2 : T(0));
    zb = z0 + (L2 > T(0) ? dz * (la + arc) / L2 : T(0));
    len = sqrt(L2 * L2 + dz * dz);
  }
  const T ax[3] = {R[2], R[5], R[8]};
  for (int k = 0; k < 3; k++) {
    t0[k] = c[k] + a2[0] * e1[k] + a2[1] * e2[k] + (type == 5 ? za * ax[k] : T(0));
    t1[k] = c[k] + b2[0] * e1[k] + b2[1] * e2[k] + (type == 5 ? zb * ax[k] : T(0));
  }
  return len;
}

}  // namespace mjbwrap
