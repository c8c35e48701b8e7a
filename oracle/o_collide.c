/*
 * Oracle (test infrastructure): broadphase + primitive narrowphase in FP64.
 * Follows the reference's pair loop (collision.hpp:235-501: bounding-sphere
 * cull, plane-X, analytic sphere/capsule-box) with MuJoCo's per-pair contact
 * rules instead of the reference's one-contact-per-pair simplification
 * (collision.hpp:310-333):
 *   plane-sphere 1, plane-capsule 2 (end caps), plane-box <= 4 (deepest
 *   corners), plane-ellipsoid/cylinder/mesh 1 (support point),
 *   sphere-sphere 1, sphere-capsule 1, capsule-capsule 1 (closest segment
 *   points), sphere-box 1, capsule-box 1 (deepest axis point, convex search),
 *   box-box <= 4 (separating axes; clipped face contacts or one edge-edge
 *   contact).
 * Contact normals point from geom1 to geom2; dist < 0 is penetration; the
 * contact position is the midpoint between the two surfaces.  The tangent
 * frame is built from the normal by projecting (0,1,0), or (0,0,1) when
 * |n_y| >= 0.5 (MuJoCo's frame rule; unverified vs MuJoCo C).
 */
#include "mjoracle.h"
#include "o_util.h"

#define ORACLE_UNSUPPORTED 16

static void make_frame(const double n_in[3], double frame[9]) {
  double n[3] = {n_in[0], n_in[1], n_in[2]};
  double l = o_norm3(n);
  if (l < 1e-12) { n[0] = 1; n[1] = 0; n[2] = 0; } else { n[0] /= l; n[1] /= l; n[2] /= l; }
  double y[3] = {0, 1, 0};
  if (!(n[1] < 0.5 && n[1] > -0.5)) { y[1] = 0; y[2] = 1; }
  double dn = o_dot3(n, y);
  double t1[3] = {y[0] - n[0] * dn, y[1] - n[1] * dn, y[2] - n[2] * dn};
  double lt = o_norm3(t1);
  t1[0] /= lt; t1[1] /= lt; t1[2] /= lt;
  double t2[3];
  o_cross(n, t1, t2);
  for (int k = 0; k < 3; k++) { frame[k] = n[k]; frame[3 + k] = t1[k]; frame[6 + k] = t2[k]; }
}

typedef struct {
  double pos[3], n[3], dist;
} Con;

/* ---------------------------------------------------------------- primitives */
static int plane_sphere(const double* pp, const double* pn, const double* c, double r, double margin, Con* out) {
  double d = (c[0] - pp[0]) * pn[0] + (c[1] - pp[1]) * pn[1] + (c[2] - pp[2]) * pn[2] - r;
  if (d >= margin) return 0;
  for (int k = 0; k < 3; k++) { out->pos[k] = c[k] - pn[k] * (r + 0.5 * d); out->n[k] = pn[k]; }
  out->dist = d;
  return 1;
}

static int plane_capsule(const double* pp, const double* pn, const double* c, const double* R, const double* sz, double margin, Con* out) {
  int n = 0;
  for (int e = 0; e < 2; e++) {
    double s = e == 0 ? sz[1] : -sz[1];
    double end[3] = {c[0] + R[2] * s, c[1] + R[5] * s, c[2] + R[8] * s};
    n += plane_sphere(pp, pn, end, sz[0], margin, out + n);
  }
  return n;
}

static int plane_box(const double* pp, const double* pn, const double* c, const double* R, const double* sz, double margin, Con* out) {
  double dist[8];
  int keep[8], nk = 0;
  for (int k = 0; k < 8; k++) {
    double l[3] = {(k & 1) ? sz[0] : -sz[0], (k & 2) ? sz[1] : -sz[1], (k & 4) ? sz[2] : -sz[2]};
    double w[3];
    o_mulmat(R, l, w);
    dist[k] = (c[0] + w[0] - pp[0]) * pn[0] + (c[1] + w[1] - pp[1]) * pn[1] + (c[2] + w[2] - pp[2]) * pn[2];
    if (dist[k] < margin) keep[nk++] = k;
  }
  /* more than four: drop the shallowest (ties keep the lower corner index) */
  while (nk > 4) {
    int worst = 0;
    for (int i = 1; i < nk; i++)
      if (dist[keep[i]] >= dist[keep[worst]]) worst = i;
    for (int i = worst; i < nk - 1; i++) keep[i] = keep[i + 1];
    nk--;
  }
  for (int i = 0; i < nk; i++) {
    int k = keep[i];
    double l[3] = {(k & 1) ? sz[0] : -sz[0], (k & 2) ? sz[1] : -sz[1], (k & 4) ? sz[2] : -sz[2]};
    double w[3];
    o_mulmat(R, l, w);
    for (int a = 0; a < 3; a++) { out[i].pos[a] = c[a] + w[a] - pn[a] * 0.5 * dist[k]; out[i].n[a] = pn[a]; }
    out[i].dist = dist[k];
  }
  return nk;
}

/* support point of a convex primitive along world direction dir */
static void support(int type, const double* c, const double* R, const double* sz, const OModel* m, int dataid, const double* dir, double* out) {
  double ld[3], lp[3] = {0, 0, 0};
  o_mulmatT(R, dir, ld);
  if (type == 2) {
    double l = o_norm3(ld);
    for (int k = 0; k < 3; k++) lp[k] = l > 1e-12 ? ld[k] / l * sz[0] : (k == 2 ? sz[0] : 0);
  } else if (type == 3) {
    double l = o_norm3(ld);
    for (int k = 0; k < 3; k++) lp[k] = l > 1e-12 ? ld[k] / l * sz[0] : 0;
    lp[2] += ld[2] >= 0 ? sz[1] : -sz[1];
  } else if (type == 4) {
    double s[3] = {sz[0] * ld[0], sz[1] * ld[1], sz[2] * ld[2]};
    double l = o_norm3(s);
    for (int k = 0; k < 3; k++) lp[k] = l > 1e-12 ? sz[k] * s[k] / l : (k == 2 ? sz[2] : 0);
  } else if (type == 5) {
    double l = sqrt(ld[0] * ld[0] + ld[1] * ld[1]);
    if (l > 1e-12) { lp[0] = ld[0] / l * sz[0]; lp[1] = ld[1] / l * sz[0]; }
    lp[2] = ld[2] >= 0 ? sz[1] : -sz[1];
  } else if (type == 6) {
    for (int k = 0; k < 3; k++) lp[k] = ld[k] >= 0 ? sz[k] : -sz[k];
  } else if (type == 7) {
    int adr = m->mesh_vertadr[dataid], n = m->mesh_vertnum[dataid];
    double best = -1e300;
    for (int v = 0; v < n; v++) {
      const double* p = &m->mesh_vert[3 * (adr + v)];
      double dd = p[0] * ld[0] + p[1] * ld[1] + p[2] * ld[2];
      if (dd > best) { best = dd; lp[0] = p[0]; lp[1] = p[1]; lp[2] = p[2]; }
    }
  }
  double w[3];
  o_mulmat(R, lp, w);
  for (int k = 0; k < 3; k++) out[k] = c[k] + w[k];
}

static int plane_convex(const double* pp, const double* pn, int type, const double* c, const double* R, const double* sz, const OModel* m, int dataid,
                        double margin, Con* out) {
  double nd[3] = {-pn[0], -pn[1], -pn[2]}, w[3];
  support(type, c, R, sz, m, dataid, nd, w);
  double d = (w[0] - pp[0]) * pn[0] + (w[1] - pp[1]) * pn[1] + (w[2] - pp[2]) * pn[2];
  if (d >= margin) return 0;
  for (int k = 0; k < 3; k++) { out->pos[k] = w[k] - pn[k] * 0.5 * d; out->n[k] = pn[k]; }
  out->dist = d;
  return 1;
}

static int sphere_sphere(const double* c1, double r1, const double* c2, double r2, double margin, Con* out) {
  double v[3] = {c2[0] - c1[0], c2[1] - c1[1], c2[2] - c1[2]};
  double l = o_norm3(v);
  double d = l - r1 - r2;
  if (d >= margin) return 0;
  double n[3];
  if (l < 1e-12) { n[0] = 1; n[1] = 0; n[2] = 0; } else { n[0] = v[0] / l; n[1] = v[1] / l; n[2] = v[2] / l; }
  for (int k = 0; k < 3; k++) { out->pos[k] = c1[k] + n[k] * (r1 + 0.5 * d); out->n[k] = n[k]; }
  out->dist = d;
  return 1;
}

static void closest_on_segment(const double* a, const double* b, const double* p, double* q) {
  double ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double l2 = o_dot3(ab, ab);
  double t = l2 > 1e-30 ? ((p[0] - a[0]) * ab[0] + (p[1] - a[1]) * ab[1] + (p[2] - a[2]) * ab[2]) / l2 : 0;
  t = t < 0 ? 0 : t > 1 ? 1 : t;
  for (int k = 0; k < 3; k++) q[k] = a[k] + t * ab[k];
}

/* closest points between segments p1q1 and p2q2 (clamped parameter method) */
static void segment_segment(const double* p1, const double* q1, const double* p2, const double* q2, double* c1, double* c2) {
  double d1[3] = {q1[0] - p1[0], q1[1] - p1[1], q1[2] - p1[2]};
  double d2[3] = {q2[0] - p2[0], q2[1] - p2[1], q2[2] - p2[2]};
  double r[3] = {p1[0] - p2[0], p1[1] - p2[1], p1[2] - p2[2]};
  double a = o_dot3(d1, d1), e = o_dot3(d2, d2), f = o_dot3(d2, r);
  double s, t;
  if (a <= 1e-30 && e <= 1e-30) { s = t = 0; }
  else if (a <= 1e-30) { s = 0; t = f / e; t = t < 0 ? 0 : t > 1 ? 1 : t; }
  else {
    double c = o_dot3(d1, r);
    if (e <= 1e-30) { t = 0; s = -c / a; s = s < 0 ? 0 : s > 1 ? 1 : s; }
    else {
      double b = o_dot3(d1, d2), den = a * e - b * b;
      if (den > 1e-12 * a * e) { s = (b * f - c * e) / den; s = s < 0 ? 0 : s > 1 ? 1 : s; }
      else s = 0.5;  /* parallel: use the midpoint of segment 1 */
      t = (b * s + f) / e;
      if (t < 0) { t = 0; s = -c / a; s = s < 0 ? 0 : s > 1 ? 1 : s; }
      else if (t > 1) { t = 1; s = (b - c) / a; s = s < 0 ? 0 : s > 1 ? 1 : s; }
    }
  }
  for (int k = 0; k < 3; k++) { c1[k] = p1[k] + s * d1[k]; c2[k] = p2[k] + t * d2[k]; }
}

/* signed distance from a box-local point to the box (outside > 0) */
static double box_sdist(const double* l, const double* h) {
  double q[3], o = 0;
  for (int k = 0; k < 3; k++) {
    q[k] = l[k] < -h[k] ? -h[k] : l[k] > h[k] ? h[k] : l[k];
    o += (l[k] - q[k]) * (l[k] - q[k]);
  }
  if (o > 0) return sqrt(o);
  double pen = h[0] - fabs(l[0]);
  for (int k = 1; k < 3; k++) {
    double p = h[k] - fabs(l[k]);
    if (p < pen) pen = p;
  }
  return -pen;
}

/* sphere (geom1) against box (geom2): normal from sphere to box */
static int sphere_box(const double* c, double r, const double* bc, const double* BR, const double* bh, double margin, Con* out) {
  double rel[3] = {c[0] - bc[0], c[1] - bc[1], c[2] - bc[2]}, lc[3], q[3];
  o_mulmatT(BR, rel, lc);
  double o2 = 0;
  for (int k = 0; k < 3; k++) {
    q[k] = lc[k] < -bh[k] ? -bh[k] : lc[k] > bh[k] ? bh[k] : lc[k];
    o2 += (lc[k] - q[k]) * (lc[k] - q[k]);
  }
  double nl[3], d;
  if (o2 > 0) {
    double l = sqrt(o2);
    for (int k = 0; k < 3; k++) nl[k] = (q[k] - lc[k]) / l;
    d = l - r;
  } else {
    int ax = 0;
    double pen = bh[0] - fabs(lc[0]);
    for (int k = 1; k < 3; k++) {
      double p = bh[k] - fabs(lc[k]);
      if (p < pen) { pen = p; ax = k; }
    }
    double sg = lc[ax] >= 0 ? 1.0 : -1.0;
    nl[0] = nl[1] = nl[2] = 0;
    nl[ax] = -sg;
    q[ax] = sg * bh[ax];
    d = -pen - r;
  }
  if (d >= margin) return 0;
  double nw[3], qw[3];
  o_mulmat(BR, nl, nw);
  o_mulmat(BR, q, qw);
  for (int k = 0; k < 3; k++) { out->n[k] = nw[k]; out->pos[k] = bc[k] + qw[k] - nw[k] * 0.5 * d; }
  out->dist = d;
  return 1;
}

static int capsule_box(const double* c, const double* R, const double* sz, const double* bc, const double* BR, const double* bh, double margin, Con* out) {
  double a0[3], a1[3];
  for (int k = 0; k < 3; k++) { a0[k] = c[k] - R[3 * k + 2] * sz[1]; a1[k] = c[k] + R[3 * k + 2] * sz[1]; }
  /* local end points */
  double r0[3] = {a0[0] - bc[0], a0[1] - bc[1], a0[2] - bc[2]}, r1[3] = {a1[0] - bc[0], a1[1] - bc[1], a1[2] - bc[2]}, l0[3], l1[3];
  o_mulmatT(BR, r0, l0);
  o_mulmatT(BR, r1, l1);
  /* exact cull: segment bounding box (box frame) outside the box inflated by
     radius + margin */
  for (int k = 0; k < 3; k++) {
    double ext = bh[k] + sz[0] + margin;
    double lo = l0[k] < l1[k] ? l0[k] : l1[k], hi = l0[k] < l1[k] ? l1[k] : l0[k];
    if (lo > ext || hi < -ext) return 0;
  }
  /* golden-section search of the convex signed distance along the axis */
  const double g = 0.6180339887498949;
  double lo = 0, hi = 1;
  double x1 = hi - g * (hi - lo), x2 = lo + g * (hi - lo), p[3];
  for (int k = 0; k < 3; k++) p[k] = l0[k] + x1 * (l1[k] - l0[k]);
  double f1 = box_sdist(p, bh);
  for (int k = 0; k < 3; k++) p[k] = l0[k] + x2 * (l1[k] - l0[k]);
  double f2 = box_sdist(p, bh);
  for (int it = 0; it < 40; it++) {
    if (f1 <= f2) {
      hi = x2; x2 = x1; f2 = f1; x1 = hi - g * (hi - lo);
      for (int k = 0; k < 3; k++) p[k] = l0[k] + x1 * (l1[k] - l0[k]);
      f1 = box_sdist(p, bh);
    } else {
      lo = x1; x1 = x2; f1 = f2; x2 = lo + g * (hi - lo);
      for (int k = 0; k < 3; k++) p[k] = l0[k] + x2 * (l1[k] - l0[k]);
      f2 = box_sdist(p, bh);
    }
  }
  double t = 0.5 * (lo + hi);
  for (int k = 0; k < 3; k++) p[k] = l0[k] + t * (l1[k] - l0[k]);
  double ft = box_sdist(p, bh);
  double fe0 = box_sdist(l0, bh), fe1 = box_sdist(l1, bh);
  if (fe0 < ft) { t = 0; ft = fe0; }
  if (fe1 < ft) { t = 1; }
  double s[3];
  for (int k = 0; k < 3; k++) s[k] = a0[k] + t * (a1[k] - a0[k]);
  return sphere_box(s, sz[0], bc, BR, bh, margin, out);
}

/* Box-box by separating axes.  The 15 axes (3 + 3 face normals, 9 edge
 * cross products) give the least-penetrating axis; a face axis is kept
 * unless an edge axis penetrates less by more than 5 % (and 1e-5 of the box
 * scale).  Face case: the incident face (the face of the other box most
 * anti-parallel to the reference normal) is clipped against the side planes
 * of the reference face; points below the reference face plus the margin
 * become contacts at the midpoint between the point and its projection,
 * reduced to at most 4 by taking the extremes along the reference face's
 * diagonals.  Edge case: one contact at the closest points of the two
 * supporting edges.  Normal from box 1 to box 2. */
static double box_radius(const double (*ax)[3], const double* h, const double* L) {
  return h[0] * fabs(o_dot3(ax[0], L)) + h[1] * fabs(o_dot3(ax[1], L)) + h[2] * fabs(o_dot3(ax[2], L));
}

static int box_box(const double* c1, const double* R1, const double* h1, const double* c2, const double* R2, const double* h2, double margin, Con* out) {
  double A[3][3], B[3][3], T[3];
  for (int k = 0; k < 3; k++)
    for (int r = 0; r < 3; r++) { A[k][r] = R1[3 * r + k]; B[k][r] = R2[3 * r + k]; }
  for (int k = 0; k < 3; k++) T[k] = c2[k] - c1[k];
  double best_face = -1e300, best_edge = -1e300, Le[3] = {0, 0, 0};
  int face = -1, ei = -1, ej = -1;
  for (int i = 0; i < 6; i++) {
    const double* L = i < 3 ? A[i] : B[i - 3];
    double dd = fabs(o_dot3(T, L)) - box_radius((const double(*)[3])A, h1, L) - box_radius((const double(*)[3])B, h2, L);
    if (dd > margin) return 0;
    if (dd > best_face) { best_face = dd; face = i; }
  }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double L[3];
      o_cross(A[i], B[j], L);
      double len = o_norm3(L);
      if (len < 1e-6) continue;
      for (int k = 0; k < 3; k++) L[k] /= len;
      double dd = fabs(o_dot3(T, L)) - box_radius((const double(*)[3])A, h1, L) - box_radius((const double(*)[3])B, h2, L);
      if (dd > margin) return 0;
      if (dd > best_edge) { best_edge = dd; ei = i; ej = j; for (int k = 0; k < 3; k++) Le[k] = L[k]; }
    }
  double scale = h1[0] + h1[1] + h1[2] + h2[0] + h2[1] + h2[2];
  if (ei >= 0 && best_edge - best_face > 0.05 * fabs(best_face) + 1e-5 * scale) {
    double L[3] = {Le[0], Le[1], Le[2]};
    if (o_dot3(T, L) < 0) for (int k = 0; k < 3; k++) L[k] = -L[k];
    double ca[3], cb[3], a0[3], a1[3], b0[3], b1[3], xa[3], xb[3];
    for (int k = 0; k < 3; k++) { ca[k] = c1[k]; cb[k] = c2[k]; }
    for (int m = 0; m < 3; m++) {
      if (m != ei) { double sg = o_dot3(A[m], L) >= 0 ? 1 : -1; for (int k = 0; k < 3; k++) ca[k] += sg * h1[m] * A[m][k]; }
      if (m != ej) { double sg = o_dot3(B[m], L) >= 0 ? 1 : -1; for (int k = 0; k < 3; k++) cb[k] -= sg * h2[m] * B[m][k]; }
    }
    for (int k = 0; k < 3; k++) {
      a0[k] = ca[k] - h1[ei] * A[ei][k]; a1[k] = ca[k] + h1[ei] * A[ei][k];
      b0[k] = cb[k] - h2[ej] * B[ej][k]; b1[k] = cb[k] + h2[ej] * B[ej][k];
    }
    segment_segment(a0, a1, b0, b1, xa, xb);
    for (int k = 0; k < 3; k++) { out->pos[k] = 0.5 * (xa[k] + xb[k]); out->n[k] = L[k]; }
    out->dist = best_edge;
    return 1;
  }
  /* face case */
  const int refA = face < 3, ax = face % 3;
  const double (*Rf)[3] = refA ? (const double(*)[3])A : (const double(*)[3])B;
  const double (*Ri)[3] = refA ? (const double(*)[3])B : (const double(*)[3])A;
  const double *cf = refA ? c1 : c2, *ci = refA ? c2 : c1, *hf = refA ? h1 : h2, *hi = refA ? h2 : h1;
  double Tri[3] = {ci[0] - cf[0], ci[1] - cf[1], ci[2] - cf[2]}, n[3];
  double sn = o_dot3(Tri, Rf[ax]) >= 0 ? 1 : -1;
  for (int k = 0; k < 3; k++) n[k] = sn * Rf[ax][k];
  int kf = 0;
  double bestk = -1;
  for (int k = 0; k < 3; k++) { double a = fabs(o_dot3(Ri[k], n)); if (a > bestk) { bestk = a; kf = k; } }
  double s = o_dot3(Ri[kf], n) > 0 ? -1 : 1;
  int k1 = (kf + 1) % 3, k2 = (kf + 2) % 3;
  double poly[16][3], tmp[16][3];
  int np = 4;
  const double sg1[4] = {1, -1, -1, 1}, sg2[4] = {1, 1, -1, -1};
  for (int v = 0; v < 4; v++)
    for (int k = 0; k < 3; k++) poly[v][k] = ci[k] + s * hi[kf] * Ri[kf][k] + sg1[v] * hi[k1] * Ri[k1][k] + sg2[v] * hi[k2] * Ri[k2][k];
  const int a1 = (ax + 1) % 3, a2 = (ax + 2) % 3;
  /* clip against (p - cf).dir <= ext for dir in {u, -u, v, -v} */
  for (int pl = 0; pl < 4 && np > 0; pl++) {
    const double* dir = pl < 2 ? Rf[a1] : Rf[a2];
    double sgn = (pl % 2) ? -1 : 1, ext = pl < 2 ? hf[a1] : hf[a2];
    int nt = 0;
    for (int v = 0; v < np; v++) {
      const double* P = poly[v];
      const double* Q = poly[(v + 1) % np];
      double dp = sgn * ((P[0] - cf[0]) * dir[0] + (P[1] - cf[1]) * dir[1] + (P[2] - cf[2]) * dir[2]) - ext;
      double dq = sgn * ((Q[0] - cf[0]) * dir[0] + (Q[1] - cf[1]) * dir[1] + (Q[2] - cf[2]) * dir[2]) - ext;
      if (dp <= 0) { for (int k = 0; k < 3; k++) tmp[nt][k] = P[k]; nt++; }
      if ((dp <= 0) != (dq <= 0)) {
        double t = dp / (dp - dq);
        for (int k = 0; k < 3; k++) tmp[nt][k] = P[k] + t * (Q[k] - P[k]);
        nt++;
      }
    }
    np = nt;
    for (int v = 0; v < np; v++) for (int k = 0; k < 3; k++) poly[v][k] = tmp[v][k];
  }
  double refc[3];
  for (int k = 0; k < 3; k++) refc[k] = cf[k] + hf[ax] * n[k];
  double pts[16][3], dep[16], uu[16], vv[16];
  int nc = 0;
  for (int v = 0; v < np; v++) {
    double dd = (poly[v][0] - refc[0]) * n[0] + (poly[v][1] - refc[1]) * n[1] + (poly[v][2] - refc[2]) * n[2];
    if (!(dd < margin)) continue;
    for (int k = 0; k < 3; k++) pts[nc][k] = poly[v][k] - 0.5 * dd * n[k];
    dep[nc] = dd;
    uu[nc] = (poly[v][0] - cf[0]) * Rf[a1][0] + (poly[v][1] - cf[1]) * Rf[a1][1] + (poly[v][2] - cf[2]) * Rf[a1][2];
    vv[nc] = (poly[v][0] - cf[0]) * Rf[a2][0] + (poly[v][1] - cf[1]) * Rf[a2][1] + (poly[v][2] - cf[2]) * Rf[a2][2];
    nc++;
  }
  int sel[4], ns = 0;
  if (nc <= 4) {
    for (int v = 0; v < nc; v++) sel[ns++] = v;
  } else {
    const double du[4] = {1, 1, -1, -1}, dv[4] = {1, -1, 1, -1};
    for (int q = 0; q < 4; q++) {
      int bi = 0;
      for (int v = 1; v < nc; v++)
        if (du[q] * uu[v] + dv[q] * vv[v] > du[q] * uu[bi] + dv[q] * vv[bi]) bi = v;
      int dup = 0;
      for (int t = 0; t < ns; t++) dup |= sel[t] == bi;
      if (!dup) sel[ns++] = bi;
    }
  }
  double nrm = refA ? 1 : -1;
  for (int t = 0; t < ns; t++) {
    for (int k = 0; k < 3; k++) { out[t].pos[k] = pts[sel[t]][k]; out[t].n[k] = nrm * n[k]; }
    out[t].dist = dep[sel[t]];
  }
  return ns;
}

/* ------------------------------------------------------------------ convex
 * General convex pairs (MuJoCo's convex collider semantics, not the
 * reference's fixed-direction penetration estimate, collision.hpp:393-487):
 * GJK distance between the shapes' cores and, when the cores overlap, EPA
 * penetration (minimum translation distance).  Spheres and capsules enter as
 * their core point / segment and their radius is added afterwards.  One
 * contact: normal from geom1 to geom2, position at the midpoint of the two
 * witness points, dist = separation (negative = penetration).  Tolerance
 * CVX_TOL absolute (MuJoCo's ccd_tolerance default 1e-6), at most
 * CVX_ITER GJK iterations and CVX_EPA_ITER EPA expansions.  Unverified
 * against MuJoCo C. */
#define CVX_TOL 1e-6
#define CVX_ITER 64
#define CVX_EPA_ITER 24
#define CVX_MAXV (CVX_EPA_ITER + 8)
#define CVX_MAXF (2 * CVX_MAXV)
#define CVX_MAXE 48   /* horizon edges per expansion */

typedef struct {
  int type, dataid;
  const double *c, *R, *sz;
  double core;          /* radius added around the core */
  double rbound;        /* bounding radius of the geom */
} Shape;

typedef struct { double w[3], a[3]; } SV;   /* Minkowski point w = a - b */

static void core_support(const OModel* m, const Shape* s, const double* dir, double* out) {
  if (s->type == 2) { memcpy(out, s->c, 3 * sizeof(double)); return; }
  if (s->type == 3) {
    double ax = s->R[2] * dir[0] + s->R[5] * dir[1] + s->R[8] * dir[2], h = ax >= 0 ? s->sz[1] : -s->sz[1];
    for (int k = 0; k < 3; k++) out[k] = s->c[k] + s->R[3 * k + 2] * h;
    return;
  }
  support(s->type, s->c, s->R, s->sz, m, s->dataid, dir, out);
}

static void mk_support(const OModel* m, const Shape* A, const Shape* B, const double* dir, SV* v) {
  double nd[3] = {-dir[0], -dir[1], -dir[2]}, b[3];
  core_support(m, A, dir, v->a);
  core_support(m, B, nd, b);
  for (int k = 0; k < 3; k++) v->w[k] = v->a[k] - b[k];
}

static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* closest point to the origin on simplex S (n points): v, barycentric lam;
 * S and lam reduced to the supporting subset.  Returns the new size. */
static int simplex_closest(SV* S, int n, double* lam, double* v) {
  if (n == 1) { lam[0] = 1; memcpy(v, S[0].w, 3 * sizeof(double)); return 1; }
  if (n == 2) {
    double e[3] = {S[1].w[0] - S[0].w[0], S[1].w[1] - S[0].w[1], S[1].w[2] - S[0].w[2]}, ee = dot3(e, e);
    double t = ee > 0 ? -dot3(S[0].w, e) / ee : 0;
    if (t <= 0) { lam[0] = 1; memcpy(v, S[0].w, 3 * sizeof(double)); return 1; }
    if (t >= 1) { S[0] = S[1]; lam[0] = 1; memcpy(v, S[0].w, 3 * sizeof(double)); return 1; }
    lam[0] = 1 - t; lam[1] = t;
    for (int k = 0; k < 3; k++) v[k] = S[0].w[k] + t * e[k];
    return 2;
  }
  if (n == 3) {
    /* closest point of triangle (A, B, C) to the origin by Voronoi regions */
    const double *A = S[0].w, *B = S[1].w, *C = S[2].w;
    double ab[3], ac[3], ap[3] = {-A[0], -A[1], -A[2]};
    for (int k = 0; k < 3; k++) { ab[k] = B[k] - A[k]; ac[k] = C[k] - A[k]; }
    double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0 && d2 <= 0) { lam[0] = 1; memcpy(v, A, 3 * sizeof(double)); return 1; }
    double bp[3] = {-B[0], -B[1], -B[2]}, d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0 && d4 <= d3) { S[0] = S[1]; lam[0] = 1; memcpy(v, S[0].w, 3 * sizeof(double)); return 1; }
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {
      double t = d1 / (d1 - d3);
      lam[0] = 1 - t; lam[1] = t;
      for (int k = 0; k < 3; k++) v[k] = A[k] + t * ab[k];
      return 2;
    }
    double cp[3] = {-C[0], -C[1], -C[2]}, d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0 && d5 <= d6) { S[0] = S[2]; lam[0] = 1; memcpy(v, S[0].w, 3 * sizeof(double)); return 1; }
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
      double t = d2 / (d2 - d6);
      S[1] = S[2];
      lam[0] = 1 - t; lam[1] = t;
      for (int k = 0; k < 3; k++) v[k] = A[k] + t * ac[k];
      return 2;
    }
    double va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
      double t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
      S[0] = S[1]; S[1] = S[2];
      lam[0] = 1 - t; lam[1] = t;
      for (int k = 0; k < 3; k++) v[k] = S[0].w[k] + t * (S[1].w[k] - S[0].w[k]);
      return 2;
    }
    double den = 1 / (va + vb + vc), sb = vb * den, sc = vc * den;
    lam[0] = 1 - sb - sc; lam[1] = sb; lam[2] = sc;
    for (int k = 0; k < 3; k++) v[k] = A[k] + ab[k] * sb + ac[k] * sc;
    return 3;
  }
  /* tetrahedron: origin inside -> 4; else the closest of the faces that
     see the origin */
  static const int F[4][4] = {{0, 1, 2, 3}, {0, 1, 3, 2}, {0, 2, 3, 1}, {1, 2, 3, 0}};
  /* a flat tetrahedron (volume below 1e-6 of its edge product) is not
     trusted to contain the origin: every face is then a candidate */
  double t1[3], t2[3], t3[3], c23[3];
  for (int k = 0; k < 3; k++) { t1[k] = S[1].w[k] - S[0].w[k]; t2[k] = S[2].w[k] - S[0].w[k]; t3[k] = S[3].w[k] - S[0].w[k]; }
  o_cross(t2, t3, c23);
  const int flat = fabs(dot3(t1, c23)) <= 1e-6 * sqrt(dot3(t1, t1) * dot3(t2, t2) * dot3(t3, t3));
  int best = -1, bn = 0;
  double bd = 1e300, bl[3], bv[3];
  SV bs[3];
  for (int f = 0; f < 4; f++) {
    const double *P0 = S[F[f][0]].w, *P1 = S[F[f][1]].w, *P2 = S[F[f][2]].w, *Q = S[F[f][3]].w;
    double e1[3], e2[3], nrm[3];
    for (int k = 0; k < 3; k++) { e1[k] = P1[k] - P0[k]; e2[k] = P2[k] - P0[k]; }
    o_cross(e1, e2, nrm);
    double so = -dot3(nrm, P0), sq = dot3(nrm, Q) - dot3(nrm, P0);
    if (!flat && so * sq >= 0) continue;   /* origin on the same side as the 4th point */
    SV T[3] = {S[F[f][0]], S[F[f][1]], S[F[f][2]]};
    double l[3], vv[3];
    int k = simplex_closest(T, 3, l, vv);
    double dd = dot3(vv, vv);
    if (dd < bd) { bd = dd; best = f; bn = k; memcpy(bl, l, sizeof(bl)); memcpy(bv, vv, sizeof(bv)); memcpy(bs, T, sizeof(bs)); }
  }
  if (best < 0) { lam[0] = lam[1] = lam[2] = lam[3] = 0.25; v[0] = v[1] = v[2] = 0; return 4; }
  for (int i = 0; i < bn; i++) { S[i] = bs[i]; lam[i] = bl[i]; }
  memcpy(v, bv, 3 * sizeof(double));
  return bn;
}

typedef struct { int v[3]; double n[3], d; int alive; } Face;

static int epa_face(const SV* V, int i, int j, int k, const double* inner, Face* f) {
  double e1[3], e2[3], n[3];
  for (int q = 0; q < 3; q++) { e1[q] = V[j].w[q] - V[i].w[q]; e2[q] = V[k].w[q] - V[i].w[q]; }
  o_cross(e1, e2, n);
  double l = o_norm3(n);
  if (l < 1e-300) return 0;
  for (int q = 0; q < 3; q++) n[q] /= l;
  double o[3] = {V[i].w[0] - inner[0], V[i].w[1] - inner[1], V[i].w[2] - inner[2]};
  if (dot3(n, o) < 0) { int t = j; j = k; k = t; for (int q = 0; q < 3; q++) n[q] = -n[q]; }
  f->v[0] = i; f->v[1] = j; f->v[2] = k;
  memcpy(f->n, n, sizeof(n));
  f->d = dot3(n, V[i].w);
  f->alive = 1;
  return 1;
}

/* penetration of overlapping cores: depth, normal A->B, witness points on
 * the core surfaces; returns 0 when the polytope could not be built */
static int epa(const OModel* m, const Shape* A, const Shape* B, SV* S, int n, double* depth, double* nrm, double* pa, double* pb) {
  SV V[CVX_MAXV];
  Face Fc[CVX_MAXF];
  int nv = n, nf = 0;
  for (int i = 0; i < n; i++) V[i] = S[i];
  /* grow a degenerate simplex into a tetrahedron */
  static const double dirs[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  for (int t = 0; nv == 1 && t < 6; t++) {
    mk_support(m, A, B, dirs[t], &V[1]);
    double e[3] = {V[1].w[0] - V[0].w[0], V[1].w[1] - V[0].w[1], V[1].w[2] - V[0].w[2]};
    if (o_norm3(e) > CVX_TOL) nv = 2;
  }
  if (nv == 2) {
    double e[3] = {V[1].w[0] - V[0].w[0], V[1].w[1] - V[0].w[1], V[1].w[2] - V[0].w[2]}, p[3], q[3];
    const double* ax = fabs(e[0]) < fabs(e[1]) ? (fabs(e[0]) < fabs(e[2]) ? dirs[0] : dirs[4]) : (fabs(e[1]) < fabs(e[2]) ? dirs[2] : dirs[4]);
    o_cross(e, ax, p);
    o_cross(e, p, q);
    const double* cand[4] = {p, q, NULL, NULL};
    double np_[3] = {-p[0], -p[1], -p[2]}, nq[3] = {-q[0], -q[1], -q[2]};
    cand[2] = np_; cand[3] = nq;
    for (int t = 0; nv == 2 && t < 4; t++) {
      mk_support(m, A, B, cand[t], &V[2]);
      double f1[3], f2[3], c[3];
      for (int k = 0; k < 3; k++) { f1[k] = V[1].w[k] - V[0].w[k]; f2[k] = V[2].w[k] - V[0].w[k]; }
      o_cross(f1, f2, c);
      if (o_norm3(c) > CVX_TOL * CVX_TOL) nv = 3;
    }
  }
  if (nv == 3) {
    double f1[3], f2[3], c[3];
    for (int k = 0; k < 3; k++) { f1[k] = V[1].w[k] - V[0].w[k]; f2[k] = V[2].w[k] - V[0].w[k]; }
    o_cross(f1, f2, c);
    for (int sg = 0; nv == 3 && sg < 2; sg++) {
      double d[3] = {sg ? -c[0] : c[0], sg ? -c[1] : c[1], sg ? -c[2] : c[2]};
      mk_support(m, A, B, d, &V[3]);
      double e3[3] = {V[3].w[0] - V[0].w[0], V[3].w[1] - V[0].w[1], V[3].w[2] - V[0].w[2]};
      if (fabs(dot3(e3, c)) > CVX_TOL * o_norm3(c)) nv = 4;
    }
  }
  if (nv < 4) return 0;
  double inner[3] = {0, 0, 0};
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 3; k++) inner[k] += 0.25 * V[i].w[k];
  static const int T4[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
  for (int f = 0; f < 4; f++)
    if (!epa_face(V, T4[f][0], T4[f][1], T4[f][2], inner, &Fc[nf])) return 0;
    else nf++;
  int best = 0;
  for (int it = 0;; it++) {
    best = -1;
    for (int f = 0; f < nf; f++)
      if (Fc[f].alive && (best < 0 || Fc[f].d < Fc[best].d)) best = f;
    if (best < 0) return 0;
    if (it >= CVX_EPA_ITER || nv >= CVX_MAXV) break;
    SV w;
    mk_support(m, A, B, Fc[best].n, &w);
    if (dot3(w.w, Fc[best].n) - Fc[best].d < CVX_TOL) break;
    /* remove the faces that see w; collect the horizon edges */
    int edges[CVX_MAXE][2], ne = 0, full = 0;
    for (int f = 0; f < nf; f++) {
      if (!Fc[f].alive) continue;
      double o[3] = {w.w[0] - V[Fc[f].v[0]].w[0], w.w[1] - V[Fc[f].v[0]].w[1], w.w[2] - V[Fc[f].v[0]].w[2]};
      if (dot3(Fc[f].n, o) <= 0) continue;
      Fc[f].alive = 0;
      for (int e = 0; e < 3; e++) {
        int a = Fc[f].v[e], b = Fc[f].v[(e + 1) % 3], found = -1;
        for (int q = 0; q < ne; q++)
          if (edges[q][0] == b && edges[q][1] == a) { found = q; break; }
        if (found >= 0) { edges[found][0] = edges[ne - 1][0]; edges[found][1] = edges[ne - 1][1]; ne--; }
        else if (ne < CVX_MAXE) { edges[ne][0] = a; edges[ne][1] = b; ne++; }
        else full = 1;
      }
    }
    if (full) {   /* horizon too long for the edge buffer: keep the polytope as it was */
      for (int f = 0; f < nf; f++) Fc[f].alive = 1;
      break;
    }
    /* compact the face list, then add the new faces */
    int k = 0;
    for (int f = 0; f < nf; f++)
      if (Fc[f].alive) Fc[k++] = Fc[f];
    nf = k;
    if (nf + ne > CVX_MAXF) break;
    V[nv] = w;
    for (int q = 0; q < ne; q++)
      if (epa_face(V, edges[q][0], edges[q][1], nv, inner, &Fc[nf])) nf++;
    nv++;
  }
  /* witness points: barycentric coordinates of d n in the closest face */
  const Face* f = &Fc[best];
  const double *P0 = V[f->v[0]].w, *P1 = V[f->v[1]].w, *P2 = V[f->v[2]].w;
  double p[3] = {f->d * f->n[0], f->d * f->n[1], f->d * f->n[2]}, e1[3], e2[3], e0[3];
  for (int q = 0; q < 3; q++) { e1[q] = P1[q] - P0[q]; e2[q] = P2[q] - P0[q]; e0[q] = p[q] - P0[q]; }
  double d00 = dot3(e1, e1), d01 = dot3(e1, e2), d11 = dot3(e2, e2), d20 = dot3(e0, e1), d21 = dot3(e0, e2);
  double den = d00 * d11 - d01 * d01, l1 = 0, l2 = 0;
  if (fabs(den) > 1e-300) { l1 = (d11 * d20 - d01 * d21) / den; l2 = (d00 * d21 - d01 * d20) / den; }
  double l0 = 1 - l1 - l2;
  for (int q = 0; q < 3; q++) {
    pa[q] = l0 * V[f->v[0]].a[q] + l1 * V[f->v[1]].a[q] + l2 * V[f->v[2]].a[q];
    pb[q] = pa[q] - p[q];
    nrm[q] = f->n[q];
  }
  *depth = f->d;
  return 1;
}

/* Newton refinement of the contact normal on curved boundaries.  Depth and
 * separation are both -min over unit n of h(n) = s(n).n, with s the support
 * of A - B; EPA's polytope approximates curved patches only coarsely and
 * GJK's duality-gap stop leaves the normal sqrt(tolerance)-accurate, so a
 * few tangent-space Newton steps on h finish the minimisation.  Each shape's
 * support is probed at n +- 1e-3 t1, t2: a shape whose support jumps there
 * (a capsule core's end switching, a box or mesh edge) has a kink across
 * the jump's tangent direction, which stays fixed; the step moves only in
 * the direction left free, with the curvature measured along it.  Two
 * independent kinks (a face, a vertex against a face) leave nothing to
 * refine.  Steps are kept only when h decreases.  *depth receives h at the
 * final normal (the support-plane distance, second-order accurate in the
 * normal), sv the support there; returns 1 when the normal moved. */
static int refine_normal(const OModel* m, const Shape* A, const Shape* B, double* n, double* depth, SV* sv) {
  int moved = 0;
  SV cur;
  mk_support(m, A, B, n, &cur);
  double h = dot3(cur.w, n);
  const double eps = 1e-3;
  for (int it = 0; it < 8; it++) {
    double t1[3], t2[3], ax[3] = {0, 0, 0};
    ax[fabs(n[0]) < 0.6 ? 0 : (fabs(n[1]) < 0.6 ? 1 : 2)] = 1;
    o_cross(n, ax, t1);
    double l = o_norm3(t1);
    for (int k = 0; k < 3; k++) t1[k] /= l;
    o_cross(n, t1, t2);
    const double* T[2] = {t1, t2};
    /* probe: per shape the largest support move and its tangent direction */
    SV pr[4];
    double jump[2] = {0, 0}, kd[2][2] = {{0, 0}, {0, 0}}, jv[2][3] = {{0, 0, 0}, {0, 0, 0}};
    for (int q = 0; q < 4; q++) {
      const double* t = T[q & 1];
      const double e = q < 2 ? eps : -eps;
      double d[3] = {n[0] + e * t[0], n[1] + e * t[1], n[2] + e * t[2]};
      mk_support(m, A, B, d, &pr[q]);
      for (int sh = 0; sh < 2; sh++) {
        double mv[3];
        for (int k = 0; k < 3; k++)
          mv[k] = sh == 0 ? pr[q].a[k] - cur.a[k] : (pr[q].a[k] - pr[q].w[k]) - (cur.a[k] - cur.w[k]);
        double lm = o_norm3(mv);
        if (lm > jump[sh]) {
          jump[sh] = lm;
          kd[sh][0] = dot3(mv, t1);
          kd[sh][1] = dot3(mv, t2);
          for (int k = 0; k < 3; k++) jv[sh][k] = mv[k] / lm;
        }
      }
    }
    const double rb[2] = {A->rbound, B->rbound};
    double free_dir[2] = {0, 0}, kink3[3] = {0, 0, 0};
    int nk = 0, blocked = 0;
    for (int sh = 0; sh < 2; sh++) {
      if (jump[sh] <= 20 * eps * rb[sh]) continue;   /* smooth: moves about eps x curvature radius */
      double lk = sqrt(kd[sh][0] * kd[sh][0] + kd[sh][1] * kd[sh][1]);
      if (lk < 0.5 * jump[sh]) { blocked = 1; continue; }   /* jump mostly along n */
      double f[2] = {-kd[sh][1] / lk, kd[sh][0] / lk};
      if (nk && fabs(f[0] * free_dir[1] - f[1] * free_dir[0]) > 0.1) blocked = 1;   /* two kinks */
      free_dir[0] = f[0];
      free_dir[1] = f[1];
      memcpy(kink3, jv[sh], sizeof(kink3));
      nk++;
    }
    if (blocked) break;
    if (nk) {
      /* the kink's minimum lies where the jumping support switches: n
         orthogonal to the jump (a segment's axis, an edge) */
      double nn[3], dn = dot3(n, kink3);
      for (int k = 0; k < 3; k++) nn[k] = n[k] - dn * kink3[k];
      double ln = o_norm3(nn);
      for (int k = 0; k < 3; k++) nn[k] /= ln;
      SV w;
      mk_support(m, A, B, nn, &w);
      double hn = dot3(w.w, nn);
      if (hn < h - 1e-15) {
        memcpy(n, nn, sizeof(nn));
        h = hn;
        cur = w;
        moved = 1;
      }
    }
    double u[2];
    if (nk == 0) {
      double H[2][2], g[2] = {dot3(cur.w, t1), dot3(cur.w, t2)};
      for (int j2 = 0; j2 < 2; j2++)
        for (int i2 = 0; i2 < 2; i2++) H[i2][j2] = (dot3(pr[j2].w, T[i2]) - dot3(pr[j2 + 2].w, T[i2])) / (2 * eps) - (i2 == j2 ? h : 0);
      double a = H[0][0], b = 0.5 * (H[0][1] + H[1][0]), c = H[1][1], det = a * c - b * b;
      if (!(a > 0 && det > 0)) break;
      u[0] = -(c * g[0] - b * g[1]) / det;
      u[1] = -(a * g[1] - b * g[0]) / det;
    } else {
      double e3[3], dp[3], dm[3];
      for (int k = 0; k < 3; k++) {
        e3[k] = free_dir[0] * t1[k] + free_dir[1] * t2[k];
        dp[k] = n[k] + eps * e3[k];
        dm[k] = n[k] - eps * e3[k];
      }
      SV sp, sm;
      mk_support(m, A, B, dp, &sp);
      mk_support(m, A, B, dm, &sm);
      double He = (dot3(sp.w, e3) - dot3(sm.w, e3)) / (2 * eps) - h, ge = dot3(cur.w, e3);
      if (!(He > 0)) break;
      u[0] = -ge / He * free_dir[0];
      u[1] = -ge / He * free_dir[1];
    }
    if (sqrt(u[0] * u[0] + u[1] * u[1]) < 1e-12) break;
    int accepted = 0;
    for (int ls = 0; ls < 4 && !accepted; ls++, u[0] *= 0.5, u[1] *= 0.5) {
      double nn[3];
      for (int k = 0; k < 3; k++) nn[k] = n[k] + u[0] * t1[k] + u[1] * t2[k];
      double ln = o_norm3(nn);
      for (int k = 0; k < 3; k++) nn[k] /= ln;
      SV w;
      mk_support(m, A, B, nn, &w);
      double hn = dot3(w.w, nn);
      if (hn < h - 1e-15) {
        memcpy(n, nn, sizeof(nn));
        h = hn;
        cur = w;
        accepted = moved = 1;
      }
    }
    if (!accepted) break;
  }
  *depth = h;   /* support-plane distance at the final normal */
  *sv = cur;
  return moved;
}

/* largest move of a shape's core support point when the direction tilts by
 * 1e-3 rad: about 1e-3 x the curvature radius where the support is unique,
 * a jump across a face or an edge where it is not */
static double support_jump(const OModel* m, const Shape* s, const double* n) {
  double t1[3], t2[3], ax[3] = {0, 0, 0}, s0[3], j = 0;
  ax[fabs(n[0]) < 0.6 ? 0 : (fabs(n[1]) < 0.6 ? 1 : 2)] = 1;
  o_cross(n, ax, t1);
  double l = o_norm3(t1);
  for (int k = 0; k < 3; k++) t1[k] /= l;
  o_cross(n, t1, t2);
  core_support(m, s, n, s0);
  for (int i = 0; i < 4; i++) {   /* +-t1, +-t2: a kink on either side shows */
    const double* t = (i & 1) ? t2 : t1;
    const double tilt = i < 2 ? 1e-3 : -1e-3;
    double d[3] = {n[0] + tilt * t[0], n[1] + tilt * t[1], n[2] + tilt * t[2]}, s1[3];
    core_support(m, s, d, s1);
    double e[3] = {s1[0] - s0[0], s1[1] - s0[1], s1[2] - s0[2]}, le = o_norm3(e);
    if (le > j) j = le;
  }
  return j;
}

/* centre of a shape's support set at direction n (a face, an edge or a
 * point): the mean of the supports along 16 directions tilted by 0.05 rad
 * around n; *spread = the largest distance of a sample from the mean */
static void support_set_center(const OModel* m, const Shape* s, const double* n, double* c, double* spread) {
  double t1[3], t2[3], ax[3] = {0, 0, 0}, p[16][3];
  ax[fabs(n[0]) < 0.6 ? 0 : (fabs(n[1]) < 0.6 ? 1 : 2)] = 1;
  o_cross(n, ax, t1);
  double l = o_norm3(t1);
  for (int k = 0; k < 3; k++) t1[k] /= l;
  o_cross(n, t1, t2);
  c[0] = c[1] = c[2] = 0;
  for (int i = 0; i < 16; i++) {
    double th = 0.39269908169872414 * i, ct = cos(th), st = sin(th), d[3];
    for (int k = 0; k < 3; k++) d[k] = n[k] + 0.05 * (ct * t1[k] + st * t2[k]);
    core_support(m, s, d, p[i]);
    for (int k = 0; k < 3; k++) c[k] += p[i][k] / 16;
  }
  *spread = 0;
  for (int i = 0; i < 16; i++) {
    double e[3] = {p[i][0] - c[0], p[i][1] - c[1], p[i][2] - c[2]}, le = o_norm3(e);
    if (le > *spread) *spread = le;
  }
}

/* Witness points (core surfaces, pb = pa + sep n): where one shape's
 * support point is unique at the normal (a curved patch, a vertex, a
 * sphere's centre) it is that shape's support point; where both touch with
 * a face or an edge the contact point is not unique: it is the centre of
 * the smaller of the two support sets (a face's or an edge's middle), a
 * choice that does not depend on how GJK / EPA reached the normal. */
static void polish_witness(const OModel* m, const Shape* A, const Shape* B, const double* n, double sep, double* pa, double* pb) {
  double nn[3] = {-n[0], -n[1], -n[2]};
  double jA = support_jump(m, A, n), jB = support_jump(m, B, nn);
  int sa = jA <= 4e-3 * A->rbound, sb = jB <= 4e-3 * B->rbound;
  if (sa && (!sb || jA <= jB)) {
    core_support(m, A, n, pa);
    for (int k = 0; k < 3; k++) pb[k] = pa[k] + sep * n[k];
  } else if (sb) {
    core_support(m, B, nn, pb);
    for (int k = 0; k < 3; k++) pa[k] = pb[k] - sep * n[k];
  } else {
    double cA[3], cB[3], sprA, sprB;
    support_set_center(m, A, n, cA, &sprA);
    support_set_center(m, B, nn, cB, &sprB);
    if (sprA <= sprB) {
      for (int k = 0; k < 3; k++) { pa[k] = cA[k]; pb[k] = cA[k] + sep * n[k]; }
    } else {
      for (int k = 0; k < 3; k++) { pb[k] = cB[k]; pa[k] = cB[k] - sep * n[k]; }
    }
  }
}

static int convex_pair(const OModel* m, const Shape* A, const Shape* B, double margin, Con* out) {
  double dir[3] = {B->c[0] - A->c[0], B->c[1] - A->c[1], B->c[2] - A->c[2]};
  if (o_norm3(dir) < 1e-12) { dir[0] = 1; dir[1] = dir[2] = 0; }
  SV S[4];
  double lam[4], v[3];
  /* GJK on the Minkowski difference A - B */
  mk_support(m, A, B, dir, &S[0]);
  int n = 1, overlap = 0;
  memcpy(v, S[0].w, sizeof(v));
  lam[0] = 1;
  for (int it = 0; it < CVX_ITER; it++) {
    double vv = dot3(v, v);
    if (vv < CVX_TOL * CVX_TOL) { overlap = 1; break; }
    double nd[3] = {-v[0], -v[1], -v[2]};
    SV w;
    mk_support(m, A, B, nd, &w);
    if (vv - dot3(v, w.w) <= CVX_TOL * sqrt(vv)) break;   /* no progress: v is the closest point */
    /* a support point already in the simplex: no progress either */
    int dup = 0;
    for (int i = 0; i < n; i++) {
      double e[3] = {w.w[0] - S[i].w[0], w.w[1] - S[i].w[1], w.w[2] - S[i].w[2]};
      if (dot3(e, e) <= 1e-16) dup = 1;
    }
    if (dup) break;
    S[n++] = w;
    n = simplex_closest(S, n, lam, v);
    if (n == 4) { overlap = 1; break; }
  }
  double pa[3] = {0, 0, 0}, pb[3] = {0, 0, 0}, nrm[3], dist;
  if (!overlap) {
    for (int i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) { pa[k] += lam[i] * S[i].a[k]; pb[k] += lam[i] * (S[i].a[k] - S[i].w[k]); }
    double len = o_norm3(v), h = -len;
    for (int k = 0; k < 3; k++) nrm[k] = -v[k] / len;
    /* the separation is -min_n h(n) too: GJK's duality-gap stop leaves the
       normal only sqrt(tolerance)-accurate on curved shapes */
    SV sv;
    if (refine_normal(m, A, B, nrm, &h, &sv))
      for (int k = 0; k < 3; k++) { pa[k] = sv.a[k]; pb[k] = sv.a[k] - sv.w[k]; }
    if (-h > 0) len = -h;
    polish_witness(m, A, B, nrm, len, pa, pb);
    dist = len - A->core - B->core;
  } else {
    double depth;
    if (!epa(m, A, B, S, n, &depth, nrm, pa, pb)) return 0;
    SV sv;
    if (refine_normal(m, A, B, nrm, &depth, &sv))
      for (int k = 0; k < 3; k++) { pa[k] = sv.a[k]; pb[k] = sv.a[k] - sv.w[k]; }
    polish_witness(m, A, B, nrm, -depth, pa, pb);
    dist = -depth - A->core - B->core;
  }
  if (!(dist < margin)) return 0;
  for (int k = 0; k < 3; k++) {
    pa[k] += A->core * nrm[k];
    pb[k] -= B->core * nrm[k];
    out->pos[k] = 0.5 * (pa[k] + pb[k]);
    out->n[k] = nrm[k];
  }
  out->dist = dist;
  return 1;
}

static int add_contacts(const OModel* m, OData* d, int pair, const Con* cs, int n) {
  const int* pi = &m->pair_int[6 * pair];
  const double* pr = &m->pair_real[16 * pair];
  for (int i = 0; i < n; i++) {
    if (d->ncon >= d->ncon_max) {
      d->ncon_dropped++;
      d->status |= ORACLE_CONTACT_OVERFLOW;
      continue;
    }
    double* c = &d->contact[ORACLE_CONTACT_STRIDE * d->ncon++];
    for (int k = 0; k < 3; k++) c[k] = cs[i].pos[k];
    make_frame(cs[i].n, c + 3);
    c[12] = cs[i].dist;
    c[13] = pair;
    c[14] = pi[0];
    c[15] = pi[1];
    c[16] = pi[4];
    c[17] = pr[2];
    c[18] = pr[0] - pr[1];
    c[19] = -1;
  }
  return n;
}

void oracle_collide(const OModel* m, OData* d) {
  d->ncon = 0;
  d->ncon_dropped = 0;
  if (m->disableflags & ((1 << 0) | (1 << 4))) return;
  for (int p = 0; p < m->npair; p++) {
    const int* pi = &m->pair_int[6 * p];
    const double* pr = &m->pair_real[16 * p];
    int g1 = pi[0], g2 = pi[1];
    int t1 = m->geom_type[g1], t2 = m->geom_type[g2];
    double margin = pr[0];
    const double *c1 = &d->geom_xpos[3 * g1], *c2 = &d->geom_xpos[3 * g2];
    const double *R1 = &d->geom_xmat[9 * g1], *R2 = &d->geom_xmat[9 * g2];
    const double *s1 = &m->geom_size[3 * g1], *s2 = &m->geom_size[3 * g2];
    Con cs[4];
    int n = 0;
    if (t1 == 0) {
      double pn[3] = {R1[2], R1[5], R1[8]};
      double rb = m->geom_rbound[g2];
      double cd = (c2[0] - c1[0]) * pn[0] + (c2[1] - c1[1]) * pn[1] + (c2[2] - c1[2]) * pn[2];
      if (rb > 0 && cd > rb + margin) continue;
      if (t2 == 2) n = plane_sphere(c1, pn, c2, s2[0], margin, cs);
      else if (t2 == 3) n = plane_capsule(c1, pn, c2, R2, s2, margin, cs);
      else if (t2 == 6) n = plane_box(c1, pn, c2, R2, s2, margin, cs);
      else if (t2 == 4 || t2 == 5 || t2 == 7) n = plane_convex(c1, pn, t2, c2, R2, s2, m, m->geom_dataid[g2], margin, cs);
      else { d->status |= ORACLE_UNSUPPORTED; continue; }
    } else {
      double v[3] = {c2[0] - c1[0], c2[1] - c1[1], c2[2] - c1[2]};
      if (o_norm3(v) > m->geom_rbound[g1] + m->geom_rbound[g2] + margin) continue;
      if (t1 == 2 && t2 == 2) n = sphere_sphere(c1, s1[0], c2, s2[0], margin, cs);
      else if (t1 == 2 && t2 == 3) {
        double a0[3], a1[3], q[3];
        for (int k = 0; k < 3; k++) { a0[k] = c2[k] - R2[3 * k + 2] * s2[1]; a1[k] = c2[k] + R2[3 * k + 2] * s2[1]; }
        closest_on_segment(a0, a1, c1, q);
        n = sphere_sphere(c1, s1[0], q, s2[0], margin, cs);
      } else if (t1 == 3 && t2 == 3) {
        double p1[3], q1[3], p2[3], q2[3], x1[3], x2[3];
        for (int k = 0; k < 3; k++) {
          p1[k] = c1[k] - R1[3 * k + 2] * s1[1]; q1[k] = c1[k] + R1[3 * k + 2] * s1[1];
          p2[k] = c2[k] - R2[3 * k + 2] * s2[1]; q2[k] = c2[k] + R2[3 * k + 2] * s2[1];
        }
        segment_segment(p1, q1, p2, q2, x1, x2);
        n = sphere_sphere(x1, s1[0], x2, s2[0], margin, cs);
      } else if (t1 == 2 && t2 == 6) n = sphere_box(c1, s1[0], c2, R2, s2, margin, cs);
      else if (t1 == 3 && t2 == 6) n = capsule_box(c1, R1, s1, c2, R2, s2, margin, cs);
      else if (t1 == 6 && t2 == 6) n = box_box(c1, R1, s1, c2, R2, s2, margin, cs);
      else if (t1 >= 2 && t2 >= 2 && t1 <= 7 && t2 <= 7) {
        Shape A = {t1, m->geom_dataid[g1], c1, R1, s1, t1 == 2 || t1 == 3 ? s1[0] : 0, m->geom_rbound[g1]};
        Shape B = {t2, m->geom_dataid[g2], c2, R2, s2, t2 == 2 || t2 == 3 ? s2[0] : 0, m->geom_rbound[g2]};
        n = convex_pair(m, &A, &B, margin, cs);
      } else { d->status |= ORACLE_UNSUPPORTED; continue; }
    }
    add_contacts(m, d, p, cs, n);
  }
}
