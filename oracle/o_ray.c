/*
 * Oracle (test infrastructure): ray casting against the geoms of one env in
 * FP64, at the poses of the last oracle_kinematics call.  Semantics follow
 * the reference's batched raycast (src/batched.cpp:1729-1893, mj_ray rules):
 * planes are hit from their +z side within positive half sizes; spheres,
 * ellipsoids, capsules, cylinders and boxes are hit (a ray starting inside a
 * box returns its exit); t is in units of the ray vector; -1 = no hit.
 */
#include <math.h>

#include "mjoracle.h"

static double quad_root(double a, double b, double c) {
  double disc = b * b - a * c;
  if (disc < 0 || fabs(a) < 1e-300) return -1;
  double sq = sqrt(disc), t0 = (-b - sq) / a, t1 = (-b + sq) / a;
  return t0 >= 0 ? t0 : (t1 >= 0 ? t1 : -1);
}

static double better(double best, double t) { return (t >= 0 && (best < 0 || t < best)) ? t : best; }

static double hit_local(int type, const double* s, const double* p, const double* v) {
  if (type == 0) {
    if (v[2] > -1e-300) return -1;
    double t = -p[2] / v[2];
    if (t < 0) return -1;
    double hx = p[0] + t * v[0], hy = p[1] + t * v[1];
    if ((s[0] > 0 && fabs(hx) > s[0]) || (s[1] > 0 && fabs(hy) > s[1])) return -1;
    return t;
  }
  if (type == 2) return quad_root(v[0] * v[0] + v[1] * v[1] + v[2] * v[2], p[0] * v[0] + p[1] * v[1] + p[2] * v[2], p[0] * p[0] + p[1] * p[1] + p[2] * p[2] - s[0] * s[0]);
  if (type == 4) {
    double ps[3], vs[3];
    for (int k = 0; k < 3; k++) { ps[k] = p[k] / s[k]; vs[k] = v[k] / s[k]; }
    return quad_root(vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2], ps[0] * vs[0] + ps[1] * vs[1] + ps[2] * vs[2], ps[0] * ps[0] + ps[1] * ps[1] + ps[2] * ps[2] - 1);
  }
  if (type == 3 || type == 5) {
    double r = s[0], h = s[1], best = -1;
    double a = v[0] * v[0] + v[1] * v[1], b = p[0] * v[0] + p[1] * v[1], c = p[0] * p[0] + p[1] * p[1] - r * r;
    double disc = b * b - a * c;
    if (a > 1e-300 && disc >= 0) {
      double sq = sqrt(disc), t0 = (-b - sq) / a, t1 = (-b + sq) / a;
      if (fabs(p[2] + t0 * v[2]) <= h) best = better(best, t0);
      if (fabs(p[2] + t1 * v[2]) <= h) best = better(best, t1);
    }
    for (int sgn = -1; sgn <= 1; sgn += 2) {
      if (type == 5) {
        if (fabs(v[2]) > 1e-300) {
          double t = (sgn * h - p[2]) / v[2], qx = p[0] + t * v[0], qy = p[1] + t * v[1];
          if (t >= 0 && qx * qx + qy * qy <= r * r) best = better(best, t);
        }
      } else {
        double pc[3] = {p[0], p[1], p[2] - sgn * h};
        double a2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2], b2 = pc[0] * v[0] + pc[1] * v[1] + pc[2] * v[2];
        double c2 = pc[0] * pc[0] + pc[1] * pc[1] + pc[2] * pc[2] - r * r, d2 = b2 * b2 - a2 * c2;
        if (d2 >= 0 && a2 > 1e-300) {
          double sq = sqrt(d2), u0 = (-b2 - sq) / a2, u1 = (-b2 + sq) / a2;
          if (sgn * (p[2] + u0 * v[2] - sgn * h) >= 0) best = better(best, u0);
          if (sgn * (p[2] + u1 * v[2] - sgn * h) >= 0) best = better(best, u1);
        }
      }
    }
    return best;
  }
  if (type == 6) {
    double tn = -1e300, tf = 1e300;
    for (int i = 0; i < 3; i++) {
      if (fabs(v[i]) < 1e-300) {
        if (fabs(p[i]) > s[i]) return -1;
      } else {
        double t0 = (-s[i] - p[i]) / v[i], t1 = (s[i] - p[i]) / v[i];
        double lo = t0 < t1 ? t0 : t1, hi = t0 < t1 ? t1 : t0;
        if (lo > tn) tn = lo;
        if (hi < tf) tf = hi;
      }
    }
    if (tn > tf || tf < 0) return -1;
    return tn >= 0 ? tn : tf;
  }
  return -1;
}

double oracle_ray(const OModel* m, const OData* d, const double* pnt, const double* vec, const int* include, int* geomid) {
  double best = -1;
  int bg = -1;
  for (int g = 0; g < m->ngeom; g++) {
    if (!include[g]) continue;
    const double* gp = &d->geom_xpos[3 * g];
    const double* R = &d->geom_xmat[9 * g];
    double dd[3] = {pnt[0] - gp[0], pnt[1] - gp[1], pnt[2] - gp[2]}, lp[3], lv[3];
    for (int k = 0; k < 3; k++) {
      lp[k] = R[k] * dd[0] + R[3 + k] * dd[1] + R[6 + k] * dd[2];
      lv[k] = R[k] * vec[0] + R[3 + k] * vec[1] + R[6 + k] * vec[2];
    }
    double t = hit_local(m->geom_type[g], &m->geom_size[3 * g], lp, lv);
    if (t >= 0 && (best < 0 || t < best)) {
      best = t;
      bg = g;
    }
  }
  if (geomid) *geomid = bg;
  return best;
}
