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
      else { d->status |= ORACLE_UNSUPPORTED; continue; }
    }
    add_contacts(m, d, p, cs, n);
  }
}
