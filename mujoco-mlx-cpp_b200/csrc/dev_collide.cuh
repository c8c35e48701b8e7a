// Device narrowphase (one lane per candidate pair).  Same contact rules as
// the CPU oracle: plane-sphere 1, plane-capsule 2, plane-box <= 4 deepest
// corners, plane-ellipsoid/cylinder/mesh 1 support point, sphere-sphere,
// sphere-capsule, capsule-capsule, sphere-box, capsule-box 1, box-box <= 4,
// every other convex pair 1 (GJK / EPA).  Reference pair
// loop: collision.hpp:235-501 (bounding-sphere cull :301-305, plane-X
// :310-332, sphere/capsule-box :347-391).
#pragma once
#include "dev_common.cuh"

namespace mjbdev {

struct DCon {
  float pos[3], n[3], dist;
};

__device__ __forceinline__ int c_plane_sphere(const float* pp, const float* pn, const float* c, float r, float margin, DCon* out) {
  float d = (c[0] - pp[0]) * pn[0] + (c[1] - pp[1]) * pn[1] + (c[2] - pp[2]) * pn[2] - r;
  if (!(d < margin)) return 0;
#pragma unroll
  for (int k = 0; k < 3; k++) { out->pos[k] = c[k] - pn[k] * (r + 0.5f * d); out->n[k] = pn[k]; }
  out->dist = d;
  return 1;
}

__device__ __forceinline__ int c_plane_capsule(const float* pp, const float* pn, const float* c, const float* R, const float* sz, float margin, DCon* out) {
  int n = 0;
  for (int e = 0; e < 2; e++) {
    float s = e == 0 ? sz[1] : -sz[1];
    float end[3] = {c[0] + R[2] * s, c[1] + R[5] * s, c[2] + R[8] * s};
    n += c_plane_sphere(pp, pn, end, sz[0], margin, out + n);
  }
  return n;
}

__device__ __forceinline__ int c_plane_box(const float* pp, const float* pn, const float* c, const float* R, const float* sz, float margin, DCon* out) {
  float dist[8];
  int keep[8], nk = 0;
  for (int k = 0; k < 8; k++) {
    float l[3] = {(k & 1) ? sz[0] : -sz[0], (k & 2) ? sz[1] : -sz[1], (k & 4) ? sz[2] : -sz[2]};
    float w[3];
    mulmat(R, l, w);
    dist[k] = (c[0] + w[0] - pp[0]) * pn[0] + (c[1] + w[1] - pp[1]) * pn[1] + (c[2] + w[2] - pp[2]) * pn[2];
    if (dist[k] < margin) keep[nk++] = k;
  }
  while (nk > 4) {
    int worst = 0;
    #pragma unroll 1
    for (int i = 1; i < nk; i++)
      if (dist[keep[i]] >= dist[keep[worst]]) worst = i;
    #pragma unroll 1
    for (int i = worst; i < nk - 1; i++) keep[i] = keep[i + 1];
    nk--;
  }
  #pragma unroll 1
  for (int i = 0; i < nk; i++) {
    int k = keep[i];
    float l[3] = {(k & 1) ? sz[0] : -sz[0], (k & 2) ? sz[1] : -sz[1], (k & 4) ? sz[2] : -sz[2]};
    float w[3];
    mulmat(R, l, w);
#pragma unroll
    for (int a = 0; a < 3; a++) { out[i].pos[a] = c[a] + w[a] - pn[a] * 0.5f * dist[k]; out[i].n[a] = pn[a]; }
    out[i].dist = dist[k];
  }
  return nk;
}

__device__ __forceinline__ void c_support(int type, const float* c, const float* R, const float* sz, const float* mesh, int nvert, const float* dir, float* out) {
  float ld[3], lp[3] = {0, 0, 0};
  mulmatT(R, dir, ld);
  if (type == 2) {
    float l = norm3(ld);
    for (int k = 0; k < 3; k++) lp[k] = l > 1e-12f ? ld[k] / l * sz[0] : (k == 2 ? sz[0] : 0.f);
  } else if (type == 3) {
    float l = norm3(ld);
    for (int k = 0; k < 3; k++) lp[k] = l > 1e-12f ? ld[k] / l * sz[0] : 0.f;
    lp[2] += ld[2] >= 0 ? sz[1] : -sz[1];
  } else if (type == 4) {
    float s[3] = {sz[0] * ld[0], sz[1] * ld[1], sz[2] * ld[2]};
    float l = norm3(s);
    for (int k = 0; k < 3; k++) lp[k] = l > 1e-12f ? sz[k] * s[k] / l : (k == 2 ? sz[2] : 0.f);
  } else if (type == 5) {
    float l = sqrtf(ld[0] * ld[0] + ld[1] * ld[1]);
    if (l > 1e-12f) { lp[0] = ld[0] / l * sz[0]; lp[1] = ld[1] / l * sz[0]; }
    lp[2] = ld[2] >= 0 ? sz[1] : -sz[1];
  } else if (type == 6) {
    for (int k = 0; k < 3; k++) lp[k] = ld[k] >= 0 ? sz[k] : -sz[k];
  } else if (type == 7) {
    float best = -3.0e38f;
    #pragma unroll 1
    for (int v = 0; v < nvert; v++) {
      float px = ldf(mesh, 3 * v), py = ldf(mesh, 3 * v + 1), pz = ldf(mesh, 3 * v + 2);
      float dd = px * ld[0] + py * ld[1] + pz * ld[2];
      if (dd > best) { best = dd; lp[0] = px; lp[1] = py; lp[2] = pz; }
    }
  }
  float w[3];
  mulmat(R, lp, w);
  for (int k = 0; k < 3; k++) out[k] = c[k] + w[k];
}

__device__ __forceinline__ int c_plane_convex(const float* pp, const float* pn, int type, const float* c, const float* R, const float* sz, const float* mesh, int nvert,
                                              float margin, DCon* out) {
  float nd[3] = {-pn[0], -pn[1], -pn[2]}, w[3];
  c_support(type, c, R, sz, mesh, nvert, nd, w);
  float d = (w[0] - pp[0]) * pn[0] + (w[1] - pp[1]) * pn[1] + (w[2] - pp[2]) * pn[2];
  if (!(d < margin)) return 0;
  for (int k = 0; k < 3; k++) { out->pos[k] = w[k] - pn[k] * 0.5f * d; out->n[k] = pn[k]; }
  out->dist = d;
  return 1;
}

__device__ __forceinline__ int c_sphere_sphere(const float* c1, float r1, const float* c2, float r2, float margin, DCon* out) {
  float v[3] = {c2[0] - c1[0], c2[1] - c1[1], c2[2] - c1[2]};
  float l = norm3(v);
  float d = l - r1 - r2;
  if (!(d < margin)) return 0;
  float n[3];
  if (l < 1e-12f) { n[0] = 1; n[1] = 0; n[2] = 0; } else { float il = 1.f / l; n[0] = v[0] * il; n[1] = v[1] * il; n[2] = v[2] * il; }
  for (int k = 0; k < 3; k++) { out->pos[k] = c1[k] + n[k] * (r1 + 0.5f * d); out->n[k] = n[k]; }
  out->dist = d;
  return 1;
}

__device__ __forceinline__ void c_closest_on_segment(const float* a, const float* b, const float* p, float* q) {
  float ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  float l2 = dot3(ab, ab);
  float t = l2 > 1e-30f ? ((p[0] - a[0]) * ab[0] + (p[1] - a[1]) * ab[1] + (p[2] - a[2]) * ab[2]) / l2 : 0.f;
  t = clampf(t, 0.f, 1.f);
  for (int k = 0; k < 3; k++) q[k] = a[k] + t * ab[k];
}

__device__ __forceinline__ void c_segment_segment(const float* p1, const float* q1, const float* p2, const float* q2, float* c1, float* c2) {
  float d1[3] = {q1[0] - p1[0], q1[1] - p1[1], q1[2] - p1[2]};
  float d2[3] = {q2[0] - p2[0], q2[1] - p2[1], q2[2] - p2[2]};
  float r[3] = {p1[0] - p2[0], p1[1] - p2[1], p1[2] - p2[2]};
  float a = dot3(d1, d1), e = dot3(d2, d2), f = dot3(d2, r);
  float s, t;
  if (a <= 1e-30f && e <= 1e-30f) { s = t = 0; }
  else if (a <= 1e-30f) { s = 0; t = clampf(f / e, 0.f, 1.f); }
  else {
    float c = dot3(d1, r);
    if (e <= 1e-30f) { t = 0; s = clampf(-c / a, 0.f, 1.f); }
    else {
      float b = dot3(d1, d2), den = a * e - b * b;
      if (den > 1e-12f * a * e) s = clampf((b * f - c * e) / den, 0.f, 1.f);
      else s = 0.5f;
      t = (b * s + f) / e;
      if (t < 0) { t = 0; s = clampf(-c / a, 0.f, 1.f); }
      else if (t > 1) { t = 1; s = clampf((b - c) / a, 0.f, 1.f); }
    }
  }
  for (int k = 0; k < 3; k++) { c1[k] = p1[k] + s * d1[k]; c2[k] = p2[k] + t * d2[k]; }
}

__device__ __forceinline__ float c_box_sdist(const float* l, const float* h) {
  float o = 0;
  for (int k = 0; k < 3; k++) {
    float q = clampf(l[k], -h[k], h[k]);
    o += (l[k] - q) * (l[k] - q);
  }
  if (o > 0) return sqrtf(o);
  float pen = h[0] - fabsf(l[0]);
  for (int k = 1; k < 3; k++) pen = fminf(pen, h[k] - fabsf(l[k]));
  return -pen;
}

__device__ __forceinline__ int c_sphere_box(const float* c, float r, const float* bc, const float* BR, const float* bh, float margin, DCon* out) {
  float rel[3] = {c[0] - bc[0], c[1] - bc[1], c[2] - bc[2]}, lc[3], q[3];
  mulmatT(BR, rel, lc);
  float o2 = 0;
  for (int k = 0; k < 3; k++) {
    q[k] = clampf(lc[k], -bh[k], bh[k]);
    o2 += (lc[k] - q[k]) * (lc[k] - q[k]);
  }
  float nl[3], d;
  if (o2 > 0) {
    float l = sqrtf(o2), il = 1.f / l;
    for (int k = 0; k < 3; k++) nl[k] = (q[k] - lc[k]) * il;
    d = l - r;
  } else {
    int ax = 0;
    float pen = bh[0] - fabsf(lc[0]);
    for (int k = 1; k < 3; k++) {
      float p = bh[k] - fabsf(lc[k]);
      if (p < pen) { pen = p; ax = k; }
    }
    float sg = lc[ax] >= 0 ? 1.f : -1.f;
    nl[0] = nl[1] = nl[2] = 0;
    nl[ax] = -sg;
    q[ax] = sg * bh[ax];
    d = -pen - r;
  }
  if (!(d < margin)) return 0;
  float nw[3], qw[3];
  mulmat(BR, nl, nw);
  mulmat(BR, q, qw);
  for (int k = 0; k < 3; k++) { out->n[k] = nw[k]; out->pos[k] = bc[k] + qw[k] - nw[k] * 0.5f * d; }
  out->dist = d;
  return 1;
}

__device__ __forceinline__ int c_capsule_box(const float* c, const float* R, const float* sz, const float* bc, const float* BR, const float* bh, float margin, DCon* out) {
  float a0[3], a1[3];
  for (int k = 0; k < 3; k++) { a0[k] = c[k] - R[3 * k + 2] * sz[1]; a1[k] = c[k] + R[3 * k + 2] * sz[1]; }
  float r0[3] = {a0[0] - bc[0], a0[1] - bc[1], a0[2] - bc[2]}, r1[3] = {a1[0] - bc[0], a1[1] - bc[1], a1[2] - bc[2]}, l0[3], l1[3];
  mulmatT(BR, r0, l0);
  mulmatT(BR, r1, l1);
  // exact cull: the segment's bounding box (box frame) separated from the box
  // inflated by radius + margin means every axis point is farther than that
#pragma unroll
  for (int k = 0; k < 3; k++) {
    float ext = bh[k] + sz[0] + margin;
    if (fminf(l0[k], l1[k]) > ext || fmaxf(l0[k], l1[k]) < -ext) return 0;
  }
  const float g = 0.6180339887498949f;
  float lo = 0, hi = 1;
  float x1 = hi - g * (hi - lo), x2 = lo + g * (hi - lo), p[3];
  for (int k = 0; k < 3; k++) p[k] = l0[k] + x1 * (l1[k] - l0[k]);
  float f1 = c_box_sdist(p, bh);
  for (int k = 0; k < 3; k++) p[k] = l0[k] + x2 * (l1[k] - l0[k]);
  float f2 = c_box_sdist(p, bh);
  for (int it = 0; it < 40; it++) {
    if (f1 <= f2) {
      hi = x2; x2 = x1; f2 = f1; x1 = hi - g * (hi - lo);
      for (int k = 0; k < 3; k++) p[k] = l0[k] + x1 * (l1[k] - l0[k]);
      f1 = c_box_sdist(p, bh);
    } else {
      lo = x1; x1 = x2; f1 = f2; x2 = lo + g * (hi - lo);
      for (int k = 0; k < 3; k++) p[k] = l0[k] + x2 * (l1[k] - l0[k]);
      f2 = c_box_sdist(p, bh);
    }
  }
  float t = 0.5f * (lo + hi);
  for (int k = 0; k < 3; k++) p[k] = l0[k] + t * (l1[k] - l0[k]);
  float ft = c_box_sdist(p, bh);
  float fe0 = c_box_sdist(l0, bh), fe1 = c_box_sdist(l1, bh);
  if (fe0 < ft) { t = 0; ft = fe0; }
  if (fe1 < ft) { t = 1; }
  float s[3];
  for (int k = 0; k < 3; k++) s[k] = a0[k] + t * (a1[k] - a0[k]);
  return c_sphere_box(s, sz[0], bc, BR, bh, margin, out);
}

// Tangent frame from the normal (same rule as the oracle).
__device__ __forceinline__ void c_make_frame(const float n_in[3], float* frame) {
  float n[3] = {n_in[0], n_in[1], n_in[2]};
  float l = norm3(n);
  if (l < 1e-12f) { n[0] = 1; n[1] = 0; n[2] = 0; } else { float il = 1.f / l; n[0] *= il; n[1] *= il; n[2] *= il; }
  float y[3] = {0, 1, 0};
  if (!(n[1] < 0.5f && n[1] > -0.5f)) { y[1] = 0; y[2] = 1; }
  float dn = dot3(n, y);
  float t1[3] = {y[0] - n[0] * dn, y[1] - n[1] * dn, y[2] - n[2] * dn};
  float lt = 1.f / norm3(t1);
  t1[0] *= lt; t1[1] *= lt; t1[2] *= lt;
  float t2[3];
  cross3(n, t1, t2);
  for (int k = 0; k < 3; k++) { frame[k] = n[k]; frame[3 + k] = t1[k]; frame[6 + k] = t2[k]; }
}

// Box-box by separating axes (the 15 face / edge-cross axes), as in the
// oracle: face axes are kept unless an edge axis penetrates less by more
// than 5 % (and 1e-5 of the box scale).  Face case: the incident face is
// clipped against the side planes of the reference face; points below the
// reference face plus the margin become contacts (midpoint between the point
// and its projection), at most 4, chosen as the extremes along the reference
// face's diagonals.  Edge case: one contact at the closest points of the two
// supporting edges.  Normal from box 1 to box 2.
__device__ __forceinline__ float box_radius(const float (*ax)[3], const float* h, const float* L) {
  return h[0] * fabsf(dot3(ax[0], L)) + h[1] * fabsf(dot3(ax[1], L)) + h[2] * fabsf(dot3(ax[2], L));
}

__device__ __noinline__ int c_box_box(const float* c1, const float* R1, const float* h1, const float* c2, const float* R2, const float* h2, float margin,
                                      DCon* out) {
  float A[3][3], B[3][3], T[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
#pragma unroll
    for (int r = 0; r < 3; r++) {
      A[k][r] = R1[3 * r + k];
      B[k][r] = R2[3 * r + k];
    }
    T[k] = c2[k] - c1[k];
  }
  float best_face = -1e30f, best_edge = -1e30f, Le[3] = {0.f, 0.f, 0.f};
  int face = -1, ei = -1, ej = -1;
#pragma unroll 1
  for (int i = 0; i < 6; i++) {
    const float* L = i < 3 ? A[i] : B[i - 3];
    const float dd = fabsf(dot3(T, L)) - box_radius(A, h1, L) - box_radius(B, h2, L);
    if (dd > margin) return 0;
    if (dd > best_face) { best_face = dd; face = i; }
  }
#pragma unroll 1
  for (int i = 0; i < 3; i++) {
#pragma unroll 1
    for (int j = 0; j < 3; j++) {
      float L[3];
      cross3(A[i], B[j], L);
      const float len = norm3(L);
      if (len < 1e-6f) continue;
      for (int k = 0; k < 3; k++) L[k] /= len;
      const float dd = fabsf(dot3(T, L)) - box_radius(A, h1, L) - box_radius(B, h2, L);
      if (dd > margin) return 0;
      if (dd > best_edge) { best_edge = dd; ei = i; ej = j; for (int k = 0; k < 3; k++) Le[k] = L[k]; }
    }
  }
  const float scale = h1[0] + h1[1] + h1[2] + h2[0] + h2[1] + h2[2];
  if (ei >= 0 && best_edge - best_face > 0.05f * fabsf(best_face) + 1e-5f * scale) {
    float L[3] = {Le[0], Le[1], Le[2]};
    if (dot3(T, L) < 0.f) for (int k = 0; k < 3; k++) L[k] = -L[k];
    float ca[3] = {c1[0], c1[1], c1[2]}, cb[3] = {c2[0], c2[1], c2[2]}, a0[3], a1[3], b0[3], b1[3], xa[3], xb[3];
    for (int m = 0; m < 3; m++) {
      if (m != ei) { const float sg = dot3(A[m], L) >= 0.f ? 1.f : -1.f; for (int k = 0; k < 3; k++) ca[k] += sg * h1[m] * A[m][k]; }
      if (m != ej) { const float sg = dot3(B[m], L) >= 0.f ? 1.f : -1.f; for (int k = 0; k < 3; k++) cb[k] -= sg * h2[m] * B[m][k]; }
    }
    for (int k = 0; k < 3; k++) {
      a0[k] = ca[k] - h1[ei] * A[ei][k]; a1[k] = ca[k] + h1[ei] * A[ei][k];
      b0[k] = cb[k] - h2[ej] * B[ej][k]; b1[k] = cb[k] + h2[ej] * B[ej][k];
    }
    c_segment_segment(a0, a1, b0, b1, xa, xb);
    for (int k = 0; k < 3; k++) { out->pos[k] = 0.5f * (xa[k] + xb[k]); out->n[k] = L[k]; }
    out->dist = best_edge;
    return 1;
  }
  const bool refA = face < 3;
  const int ax = face % 3;
  const float (*Rf)[3] = refA ? A : B;
  const float (*Ri)[3] = refA ? B : A;
  const float *cf = refA ? c1 : c2, *ci = refA ? c2 : c1, *hf = refA ? h1 : h2, *hi = refA ? h2 : h1;
  const float Tri[3] = {ci[0] - cf[0], ci[1] - cf[1], ci[2] - cf[2]};
  const float sn = dot3(Tri, Rf[ax]) >= 0.f ? 1.f : -1.f;
  const float n[3] = {sn * Rf[ax][0], sn * Rf[ax][1], sn * Rf[ax][2]};
  int kf = 0;
  float bestk = -1.f;
  for (int k = 0; k < 3; k++) { const float a = fabsf(dot3(Ri[k], n)); if (a > bestk) { bestk = a; kf = k; } }
  const float s = dot3(Ri[kf], n) > 0.f ? -1.f : 1.f;
  const int k1 = (kf + 1) % 3, k2 = (kf + 2) % 3;
  float poly[8][3], tmp[8][3];
  int np = 4;
  const float sg1[4] = {1.f, -1.f, -1.f, 1.f}, sg2[4] = {1.f, 1.f, -1.f, -1.f};
  for (int v = 0; v < 4; v++)
    for (int k = 0; k < 3; k++) poly[v][k] = ci[k] + s * hi[kf] * Ri[kf][k] + sg1[v] * hi[k1] * Ri[k1][k] + sg2[v] * hi[k2] * Ri[k2][k];
  const int a1 = (ax + 1) % 3, a2 = (ax + 2) % 3;
#pragma unroll 1
  for (int pl = 0; pl < 4 && np > 0; pl++) {
    const float* dir = pl < 2 ? Rf[a1] : Rf[a2];
    const float sgn = (pl % 2) ? -1.f : 1.f, ext = pl < 2 ? hf[a1] : hf[a2];
    int nt = 0;
#pragma unroll 1
    for (int v = 0; v < np; v++) {
      const float* P = poly[v];
      const float* Q = poly[(v + 1) % np];
      const float dp = sgn * ((P[0] - cf[0]) * dir[0] + (P[1] - cf[1]) * dir[1] + (P[2] - cf[2]) * dir[2]) - ext;
      const float dq = sgn * ((Q[0] - cf[0]) * dir[0] + (Q[1] - cf[1]) * dir[1] + (Q[2] - cf[2]) * dir[2]) - ext;
      if (dp <= 0.f && nt < 8) { for (int k = 0; k < 3; k++) tmp[nt][k] = P[k]; nt++; }
      if ((dp <= 0.f) != (dq <= 0.f) && nt < 8) {
        const float t = dp / (dp - dq);
        for (int k = 0; k < 3; k++) tmp[nt][k] = P[k] + t * (Q[k] - P[k]);
        nt++;
      }
    }
    np = nt;
    for (int v = 0; v < np; v++)
      for (int k = 0; k < 3; k++) poly[v][k] = tmp[v][k];
  }
  const float refc[3] = {cf[0] + hf[ax] * n[0], cf[1] + hf[ax] * n[1], cf[2] + hf[ax] * n[2]};
  float dep[8], uu[8], vv[8];
  int idx[8], nc = 0;
  for (int v = 0; v < np; v++) {
    const float dd = (poly[v][0] - refc[0]) * n[0] + (poly[v][1] - refc[1]) * n[1] + (poly[v][2] - refc[2]) * n[2];
    if (!(dd < margin)) continue;
    dep[nc] = dd;
    uu[nc] = (poly[v][0] - cf[0]) * Rf[a1][0] + (poly[v][1] - cf[1]) * Rf[a1][1] + (poly[v][2] - cf[2]) * Rf[a1][2];
    vv[nc] = (poly[v][0] - cf[0]) * Rf[a2][0] + (poly[v][1] - cf[1]) * Rf[a2][1] + (poly[v][2] - cf[2]) * Rf[a2][2];
    idx[nc] = v;
    nc++;
  }
  int sel[4], ns = 0;
  if (nc <= 4) {
    for (int v = 0; v < nc; v++) sel[ns++] = v;
  } else {
    const float du[4] = {1.f, 1.f, -1.f, -1.f}, dv[4] = {1.f, -1.f, 1.f, -1.f};
    for (int q = 0; q < 4; q++) {
      int bi = 0;
      for (int v = 1; v < nc; v++)
        if (du[q] * uu[v] + dv[q] * vv[v] > du[q] * uu[bi] + dv[q] * vv[bi]) bi = v;
      bool dup = false;
      for (int t = 0; t < ns; t++) dup |= sel[t] == bi;
      if (!dup) sel[ns++] = bi;
    }
  }
  const float nrm = refA ? 1.f : -1.f;
  for (int t = 0; t < ns; t++) {
    const int v = idx[sel[t]];
    const float dd = dep[sel[t]];
    for (int k = 0; k < 3; k++) {
      out[t].pos[k] = poly[v][k] - 0.5f * dd * n[k];
      out[t].n[k] = nrm * n[k];
    }
    out[t].dist = dd;
  }
  return ns;
}

// ------------------------------------------------------------------ convex
// General convex pairs (MuJoCo's convex collider semantics; the reference
// estimates penetration from 14 fixed directions, collision.hpp:393-487):
// GJK distance between the shapes' cores; when the cores overlap, EPA on the
// Minkowski difference and a Newton refinement of the normal on curved
// boundaries.  Spheres and capsules enter as their core point / segment and
// add their radius afterwards.  One contact: normal geom1 -> geom2, position
// at the midpoint of the witness points.  One lane per pair; the polytope
// lives in the lane's local memory (about 3 KB).
#define CVX_TOL 1e-6f
#define CVX_ITER 64
#define CVX_EPA_ITER 24
#define CVX_MAXV (CVX_EPA_ITER + 8)
#define CVX_MAXF (2 * CVX_MAXV)
#define CVX_MAXE 48

struct CShape {
  int type, nvert;
  const float *c, *R, *sz, *mesh;
  float core, rbound;
};
struct CSV { float w[3], a[3]; };
struct CFace { int v[3]; float n[3], d; };

__device__ __forceinline__ void cvx_core_support(const CShape& s, const float* dir, float* out) {
  if (s.type == 2) { for (int k = 0; k < 3; k++) out[k] = s.c[k]; return; }
  if (s.type == 3) {
    const float ax = s.R[2] * dir[0] + s.R[5] * dir[1] + s.R[8] * dir[2], h = ax >= 0.f ? s.sz[1] : -s.sz[1];
    for (int k = 0; k < 3; k++) out[k] = s.c[k] + s.R[3 * k + 2] * h;
    return;
  }
  c_support(s.type, s.c, s.R, s.sz, s.mesh, s.nvert, dir, out);
}

__device__ __forceinline__ void cvx_support(const CShape& A, const CShape& B, const float* dir, CSV& v) {
  const float nd[3] = {-dir[0], -dir[1], -dir[2]};
  float b[3];
  cvx_core_support(A, dir, v.a);
  cvx_core_support(B, nd, b);
  for (int k = 0; k < 3; k++) v.w[k] = v.a[k] - b[k];
}

// closest point of triangle S[0..2] to the origin (Voronoi regions); S and
// lam reduced to the supporting subset; returns its size
__device__ int cvx_triangle(CSV* S, float* lam, float* v) {
  const float *A = S[0].w, *B = S[1].w, *C = S[2].w;
  float ab[3], ac[3];
  for (int k = 0; k < 3; k++) { ab[k] = B[k] - A[k]; ac[k] = C[k] - A[k]; }
  const float ap[3] = {-A[0], -A[1], -A[2]};
  const float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0.f && d2 <= 0.f) { lam[0] = 1.f; for (int k = 0; k < 3; k++) v[k] = A[k]; return 1; }
  const float bp[3] = {-B[0], -B[1], -B[2]};
  const float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0.f && d4 <= d3) { S[0] = S[1]; lam[0] = 1.f; for (int k = 0; k < 3; k++) v[k] = S[0].w[k]; return 1; }
  const float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
    const float t = d1 / (d1 - d3);
    lam[0] = 1.f - t; lam[1] = t;
    for (int k = 0; k < 3; k++) v[k] = A[k] + t * ab[k];
    return 2;
  }
  const float cp[3] = {-C[0], -C[1], -C[2]};
  const float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0.f && d5 <= d6) { S[0] = S[2]; lam[0] = 1.f; for (int k = 0; k < 3; k++) v[k] = S[0].w[k]; return 1; }
  const float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
    const float t = d2 / (d2 - d6);
    for (int k = 0; k < 3; k++) v[k] = A[k] + t * ac[k];
    S[1] = S[2];
    lam[0] = 1.f - t; lam[1] = t;
    return 2;
  }
  const float va = d3 * d6 - d5 * d4;
  if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
    const float t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    S[0] = S[1]; S[1] = S[2];
    lam[0] = 1.f - t; lam[1] = t;
    for (int k = 0; k < 3; k++) v[k] = S[0].w[k] + t * (S[1].w[k] - S[0].w[k]);
    return 2;
  }
  const float den = 1.f / (va + vb + vc), sb = vb * den, sc = vc * den;
  lam[0] = 1.f - sb - sc; lam[1] = sb; lam[2] = sc;
  for (int k = 0; k < 3; k++) v[k] = A[k] + ab[k] * sb + ac[k] * sc;
  return 3;
}

// closest point of simplex S (n points) to the origin; returns the reduced
// size, 4 when the tetrahedron contains the origin
__device__ int cvx_closest(CSV* S, int n, float* lam, float* v) {
  if (n == 1) { lam[0] = 1.f; for (int k = 0; k < 3; k++) v[k] = S[0].w[k]; return 1; }
  if (n == 2) {
    float e[3];
    for (int k = 0; k < 3; k++) e[k] = S[1].w[k] - S[0].w[k];
    const float ee = dot3(e, e), t = ee > 0.f ? -dot3(S[0].w, e) / ee : 0.f;
    if (t <= 0.f) { lam[0] = 1.f; for (int k = 0; k < 3; k++) v[k] = S[0].w[k]; return 1; }
    if (t >= 1.f) { S[0] = S[1]; lam[0] = 1.f; for (int k = 0; k < 3; k++) v[k] = S[0].w[k]; return 1; }
    lam[0] = 1.f - t; lam[1] = t;
    for (int k = 0; k < 3; k++) v[k] = S[0].w[k] + t * e[k];
    return 2;
  }
  if (n == 3) return cvx_triangle(S, lam, v);
  const int F[4][4] = {{0, 1, 2, 3}, {0, 1, 3, 2}, {0, 2, 3, 1}, {1, 2, 3, 0}};
  // a flat tetrahedron (volume below 1e-6 of its edge product) cannot be
  // trusted to contain the origin: every face is then a candidate
  float t1[3], t2[3], t3[3], c23[3];
  for (int k = 0; k < 3; k++) { t1[k] = S[1].w[k] - S[0].w[k]; t2[k] = S[2].w[k] - S[0].w[k]; t3[k] = S[3].w[k] - S[0].w[k]; }
  cross3(t2, t3, c23);
  const bool flat = fabsf(dot3(t1, c23)) <= 1e-6f * norm3(t1) * norm3(t2) * norm3(t3);
  int best = -1, bn = 0;
  float bd = 3.0e38f, bl[3], bv[3];
  CSV bs[3];
  for (int f = 0; f < 4; f++) {
    const float *P0 = S[F[f][0]].w, *P1 = S[F[f][1]].w, *P2 = S[F[f][2]].w, *Q = S[F[f][3]].w;
    float e1[3], e2[3], nrm[3];
    for (int k = 0; k < 3; k++) { e1[k] = P1[k] - P0[k]; e2[k] = P2[k] - P0[k]; }
    cross3(e1, e2, nrm);
    const float so = -dot3(nrm, P0), sq = dot3(nrm, Q) - dot3(nrm, P0);
    if (!flat && so * sq >= 0.f) continue;
    CSV T[3] = {S[F[f][0]], S[F[f][1]], S[F[f][2]]};
    float l[3], vv[3];
    const int k = cvx_triangle(T, l, vv);
    const float dd = dot3(vv, vv);
    if (dd < bd) {
      bd = dd; best = f; bn = k;
      for (int q = 0; q < 3; q++) { bl[q] = l[q]; bv[q] = vv[q]; bs[q] = T[q]; }
    }
  }
  if (best < 0) { lam[0] = lam[1] = lam[2] = lam[3] = 0.25f; v[0] = v[1] = v[2] = 0.f; return 4; }
  for (int i = 0; i < bn; i++) { S[i] = bs[i]; lam[i] = bl[i]; }
  for (int k = 0; k < 3; k++) v[k] = bv[k];
  return bn;
}

__device__ __forceinline__ bool cvx_face(const CSV* V, int i, int j, int k, const float* inner, CFace& f) {
  float e1[3], e2[3], n[3];
  for (int q = 0; q < 3; q++) { e1[q] = V[j].w[q] - V[i].w[q]; e2[q] = V[k].w[q] - V[i].w[q]; }
  cross3(e1, e2, n);
  const float l = norm3(n);
  if (!(l > 1e-30f)) return false;
  for (int q = 0; q < 3; q++) n[q] /= l;
  const float o[3] = {V[i].w[0] - inner[0], V[i].w[1] - inner[1], V[i].w[2] - inner[2]};
  if (dot3(n, o) < 0.f) { const int t = j; j = k; k = t; for (int q = 0; q < 3; q++) n[q] = -n[q]; }
  f.v[0] = i; f.v[1] = j; f.v[2] = k;
  for (int q = 0; q < 3; q++) f.n[q] = n[q];
  f.d = dot3(n, V[i].w);
  return true;
}

// EPA on overlapping cores: depth, normal A -> B, core witness points
__device__ __noinline__ bool cvx_epa(const CShape& A, const CShape& B, const CSV* S, int n, float& depth, float* nrm, float* pa, float* pb) {
  CSV V[CVX_MAXV];
  CFace Fc[CVX_MAXF];
  bool alive[CVX_MAXF];
  int nv = n, nf = 0;
  for (int i = 0; i < n; i++) V[i] = S[i];
  const float dirs[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  for (int t = 0; nv == 1 && t < 6; t++) {
    cvx_support(A, B, dirs[t], V[1]);
    const float e[3] = {V[1].w[0] - V[0].w[0], V[1].w[1] - V[0].w[1], V[1].w[2] - V[0].w[2]};
    if (norm3(e) > CVX_TOL) nv = 2;
  }
  if (nv == 2) {
    const float e[3] = {V[1].w[0] - V[0].w[0], V[1].w[1] - V[0].w[1], V[1].w[2] - V[0].w[2]};
    const float* ax = fabsf(e[0]) < fabsf(e[1]) ? (fabsf(e[0]) < fabsf(e[2]) ? dirs[0] : dirs[4]) : (fabsf(e[1]) < fabsf(e[2]) ? dirs[2] : dirs[4]);
    float p[3], q[3];
    cross3(e, ax, p);
    cross3(e, p, q);
    for (int t = 0; nv == 2 && t < 4; t++) {
      const float sg = t < 2 ? 1.f : -1.f;
      const float* b = (t & 1) ? q : p;
      const float d[3] = {sg * b[0], sg * b[1], sg * b[2]};
      cvx_support(A, B, d, V[2]);
      float f1[3], f2[3], c[3];
      for (int k = 0; k < 3; k++) { f1[k] = V[1].w[k] - V[0].w[k]; f2[k] = V[2].w[k] - V[0].w[k]; }
      cross3(f1, f2, c);
      if (norm3(c) > CVX_TOL * CVX_TOL) nv = 3;
    }
  }
  if (nv == 3) {
    float f1[3], f2[3], c[3];
    for (int k = 0; k < 3; k++) { f1[k] = V[1].w[k] - V[0].w[k]; f2[k] = V[2].w[k] - V[0].w[k]; }
    cross3(f1, f2, c);
    for (int sg = 0; nv == 3 && sg < 2; sg++) {
      const float d[3] = {sg ? -c[0] : c[0], sg ? -c[1] : c[1], sg ? -c[2] : c[2]};
      cvx_support(A, B, d, V[3]);
      const float e3[3] = {V[3].w[0] - V[0].w[0], V[3].w[1] - V[0].w[1], V[3].w[2] - V[0].w[2]};
      if (fabsf(dot3(e3, c)) > CVX_TOL * norm3(c)) nv = 4;
    }
  }
  if (nv < 4) return false;
  float inner[3] = {0.f, 0.f, 0.f};
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 3; k++) inner[k] += 0.25f * V[i].w[k];
  const int T4[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
  for (int f = 0; f < 4; f++) {
    if (!cvx_face(V, T4[f][0], T4[f][1], T4[f][2], inner, Fc[nf])) return false;
    alive[nf++] = true;
  }
  int best = 0;
  #pragma unroll 1
  for (int it = 0;; it++) {
    best = -1;
    for (int f = 0; f < nf; f++)
      if (alive[f] && (best < 0 || Fc[f].d < Fc[best].d)) best = f;
    if (best < 0) return false;
    if (it >= CVX_EPA_ITER || nv >= CVX_MAXV) break;
    CSV w;
    cvx_support(A, B, Fc[best].n, w);
    if (dot3(w.w, Fc[best].n) - Fc[best].d < CVX_TOL) break;
    int edges[CVX_MAXE][2], ne = 0;
    bool full = false;
    #pragma unroll 1
    for (int f = 0; f < nf; f++) {
      if (!alive[f]) continue;
      const float* p0 = V[Fc[f].v[0]].w;
      const float o[3] = {w.w[0] - p0[0], w.w[1] - p0[1], w.w[2] - p0[2]};
      if (dot3(Fc[f].n, o) <= 0.f) continue;
      alive[f] = false;
      for (int e = 0; e < 3; e++) {
        const int a = Fc[f].v[e], b = Fc[f].v[(e + 1) % 3];
        int found = -1;
        for (int q = 0; q < ne; q++)
          if (edges[q][0] == b && edges[q][1] == a) { found = q; break; }
        if (found >= 0) { edges[found][0] = edges[ne - 1][0]; edges[found][1] = edges[ne - 1][1]; ne--; }
        else if (ne < CVX_MAXE) { edges[ne][0] = a; edges[ne][1] = b; ne++; }
        else full = true;
      }
    }
    if (full) {
      for (int f = 0; f < nf; f++) alive[f] = true;
      break;
    }
    int k = 0;
    for (int f = 0; f < nf; f++)
      if (alive[f]) { Fc[k] = Fc[f]; alive[k] = true; k++; }
    nf = k;
    if (nf + ne > CVX_MAXF) break;
    V[nv] = w;
    for (int q = 0; q < ne; q++)
      if (cvx_face(V, edges[q][0], edges[q][1], nv, inner, Fc[nf])) alive[nf++] = true;
    nv++;
  }
  const CFace& f = Fc[best];
  const float *P0 = V[f.v[0]].w, *P1 = V[f.v[1]].w, *P2 = V[f.v[2]].w;
  const float p[3] = {f.d * f.n[0], f.d * f.n[1], f.d * f.n[2]};
  float e1[3], e2[3], e0[3];
  for (int q = 0; q < 3; q++) { e1[q] = P1[q] - P0[q]; e2[q] = P2[q] - P0[q]; e0[q] = p[q] - P0[q]; }
  const float d00 = dot3(e1, e1), d01 = dot3(e1, e2), d11 = dot3(e2, e2), d20 = dot3(e0, e1), d21 = dot3(e0, e2);
  const float den = d00 * d11 - d01 * d01;
  float l1 = 0.f, l2 = 0.f;
  if (fabsf(den) > 1e-30f) { l1 = (d11 * d20 - d01 * d21) / den; l2 = (d00 * d21 - d01 * d20) / den; }
  const float l0 = 1.f - l1 - l2;
  for (int q = 0; q < 3; q++) {
    pa[q] = l0 * V[f.v[0]].a[q] + l1 * V[f.v[1]].a[q] + l2 * V[f.v[2]].a[q];
    pb[q] = pa[q] - p[q];
    nrm[q] = f.n[q];
  }
  depth = f.d;
  return true;
}

// Newton refinement of the contact normal on curved boundaries: depth and
// separation are both -min over unit n of h(n) = s(n).n (s: support of
// A - B).  Each shape's support is probed at n +- 1e-3 t1, t2; a shape whose
// support jumps (capsule core end, box or mesh edge) has a kink there: the
// normal snaps onto the kink plane (orthogonal to the jump) and Newton moves
// it only in the direction left free.  Two kinks leave nothing to refine;
// steps are kept only when h decreases.  depth receives h at the final
// normal (support-plane distance), sv the support there; returns true when
// the normal moved.
__device__ __noinline__ bool cvx_refine(const CShape& A, const CShape& B, float* n, float& depth, CSV& sv) {
  bool moved = false;
  CSV cur;
  cvx_support(A, B, n, cur);
  float h = dot3(cur.w, n);
  const float eps = 1e-3f;
  #pragma unroll 1
  for (int it = 0; it < 8; it++) {
    float t1[3], t2[3], ax[3] = {0.f, 0.f, 0.f};
    ax[fabsf(n[0]) < 0.6f ? 0 : (fabsf(n[1]) < 0.6f ? 1 : 2)] = 1.f;
    cross3(n, ax, t1);
    const float l = norm3(t1);
    for (int k = 0; k < 3; k++) t1[k] /= l;
    cross3(n, t1, t2);
    // probe: per shape the largest support move and its direction
    float prw[4][3];
    float jump[2] = {0.f, 0.f}, kd[2][2] = {{0.f, 0.f}, {0.f, 0.f}}, jv[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    #pragma unroll 1
    for (int q = 0; q < 4; q++) {
      const float* t = (q & 1) ? t2 : t1;
      const float e = q < 2 ? eps : -eps;
      const float d[3] = {n[0] + e * t[0], n[1] + e * t[1], n[2] + e * t[2]};
      CSV p;
      cvx_support(A, B, d, p);
      for (int k = 0; k < 3; k++) prw[q][k] = p.w[k];
      for (int sh = 0; sh < 2; sh++) {
        float mv[3];
        for (int k = 0; k < 3; k++) mv[k] = sh == 0 ? p.a[k] - cur.a[k] : (p.a[k] - p.w[k]) - (cur.a[k] - cur.w[k]);
        const float lm = norm3(mv);
        if (lm > jump[sh]) {
          jump[sh] = lm;
          kd[sh][0] = dot3(mv, t1);
          kd[sh][1] = dot3(mv, t2);
          for (int k = 0; k < 3; k++) jv[sh][k] = mv[k] / lm;
        }
      }
    }
    const float rb[2] = {A.rbound, B.rbound};
    float free_dir[2] = {0.f, 0.f}, kink3[3] = {0.f, 0.f, 0.f};
    int nk = 0;
    bool blocked = false;
    for (int sh = 0; sh < 2; sh++) {
      if (jump[sh] <= 20.f * eps * rb[sh]) continue;   // smooth
      const float lk = sqrtf(kd[sh][0] * kd[sh][0] + kd[sh][1] * kd[sh][1]);
      if (lk < 0.5f * jump[sh]) { blocked = true; continue; }
      const float f[2] = {-kd[sh][1] / lk, kd[sh][0] / lk};
      if (nk && fabsf(f[0] * free_dir[1] - f[1] * free_dir[0]) > 0.1f) blocked = true;
      free_dir[0] = f[0];
      free_dir[1] = f[1];
      for (int k = 0; k < 3; k++) kink3[k] = jv[sh][k];
      nk++;
    }
    if (blocked) break;
    if (nk) {
      float nn[3];
      const float dn = dot3(n, kink3);
      for (int k = 0; k < 3; k++) nn[k] = n[k] - dn * kink3[k];
      const float ln = norm3(nn);
      for (int k = 0; k < 3; k++) nn[k] /= ln;
      CSV w;
      cvx_support(A, B, nn, w);
      const float hn = dot3(w.w, nn);
      if (hn < h) {
        for (int k = 0; k < 3; k++) n[k] = nn[k];
        h = hn;
        cur = w;
        moved = true;
      }
    }
    float u[2];
    if (nk == 0) {
      const float g[2] = {dot3(cur.w, t1), dot3(cur.w, t2)};
      float H[2][2];
      for (int j2 = 0; j2 < 2; j2++) {
        H[0][j2] = (dot3(prw[j2], t1) - dot3(prw[j2 + 2], t1)) / (2.f * eps) - (j2 == 0 ? h : 0.f);
        H[1][j2] = (dot3(prw[j2], t2) - dot3(prw[j2 + 2], t2)) / (2.f * eps) - (j2 == 1 ? h : 0.f);
      }
      const float a = H[0][0], b = 0.5f * (H[0][1] + H[1][0]), c = H[1][1], det = a * c - b * b;
      if (!(a > 0.f && det > 0.f)) break;
      u[0] = -(c * g[0] - b * g[1]) / det;
      u[1] = -(a * g[1] - b * g[0]) / det;
    } else {
      float e3[3], dp[3], dm[3];
      for (int k = 0; k < 3; k++) {
        e3[k] = free_dir[0] * t1[k] + free_dir[1] * t2[k];
        dp[k] = n[k] + eps * e3[k];
        dm[k] = n[k] - eps * e3[k];
      }
      CSV sp, sm;
      cvx_support(A, B, dp, sp);
      cvx_support(A, B, dm, sm);
      const float He = (dot3(sp.w, e3) - dot3(sm.w, e3)) / (2.f * eps) - h, ge = dot3(cur.w, e3);
      if (!(He > 0.f)) break;
      u[0] = -ge / He * free_dir[0];
      u[1] = -ge / He * free_dir[1];
    }
    if (sqrtf(u[0] * u[0] + u[1] * u[1]) < 1e-12f) break;
    bool accepted = false;
    for (int ls = 0; ls < 4 && !accepted; ls++, u[0] *= 0.5f, u[1] *= 0.5f) {
      float nn[3];
      for (int k = 0; k < 3; k++) nn[k] = n[k] + u[0] * t1[k] + u[1] * t2[k];
      const float ln = norm3(nn);
      for (int k = 0; k < 3; k++) nn[k] /= ln;
      CSV w;
      cvx_support(A, B, nn, w);
      const float hn = dot3(w.w, nn);
      if (hn < h) {
        for (int k = 0; k < 3; k++) n[k] = nn[k];
        h = hn;
        cur = w;
        accepted = moved = true;
      }
    }
    if (!accepted) break;
  }
  depth = h;   // support-plane distance at the final normal
  sv = cur;
  return moved;
}

// largest move of a core support point when the direction tilts by 1e-3
// rad (small and smooth on curved patches, a jump across faces and edges)
__device__ float cvx_jump(const CShape& s, const float* n) {
  float t1[3], t2[3], ax[3] = {0.f, 0.f, 0.f}, s0[3], j = 0.f;
  ax[fabsf(n[0]) < 0.6f ? 0 : (fabsf(n[1]) < 0.6f ? 1 : 2)] = 1.f;
  cross3(n, ax, t1);
  const float l = norm3(t1);
  for (int k = 0; k < 3; k++) t1[k] /= l;
  cross3(n, t1, t2);
  cvx_core_support(s, n, s0);
  for (int i = 0; i < 4; i++) {   // +-t1, +-t2: a kink on either side shows
    const float* t = (i & 1) ? t2 : t1;
    const float tilt = i < 2 ? 1e-3f : -1e-3f;
    const float d[3] = {n[0] + tilt * t[0], n[1] + tilt * t[1], n[2] + tilt * t[2]};
    float s1[3];
    cvx_core_support(s, d, s1);
    const float e[3] = {s1[0] - s0[0], s1[1] - s0[1], s1[2] - s0[2]};
    j = fmaxf(j, norm3(e));
  }
  return j;
}

// centre of a shape's support set at direction n: mean of the supports
// along 16 directions tilted by 0.05 rad around n; spread = largest
// distance of a sample from the mean
__device__ void cvx_set_center(const CShape& s, const float* n, float* c, float& spread) {
  float t1[3], t2[3], ax[3] = {0.f, 0.f, 0.f}, p[16][3];
  ax[fabsf(n[0]) < 0.6f ? 0 : (fabsf(n[1]) < 0.6f ? 1 : 2)] = 1.f;
  cross3(n, ax, t1);
  const float l = norm3(t1);
  for (int k = 0; k < 3; k++) t1[k] /= l;
  cross3(n, t1, t2);
  c[0] = c[1] = c[2] = 0.f;
  #pragma unroll 1
  for (int i = 0; i < 16; i++) {
    float st, ct;
    sincosf(0.39269908169872414f * i, &st, &ct);
    float d[3];
    for (int k = 0; k < 3; k++) d[k] = n[k] + 0.05f * (ct * t1[k] + st * t2[k]);
    cvx_core_support(s, d, p[i]);
    for (int k = 0; k < 3; k++) c[k] += p[i][k] * (1.f / 16.f);
  }
  spread = 0.f;
  for (int i = 0; i < 16; i++) {
    const float e[3] = {p[i][0] - c[0], p[i][1] - c[1], p[i][2] - c[2]};
    spread = fmaxf(spread, norm3(e));
  }
}

// witness points with pb = pa + sep n: the support point of the shape whose
// support is unique at the normal; for face / edge against face / edge the
// centre of the smaller support set
__device__ __noinline__ void cvx_polish(const CShape& A, const CShape& B, const float* n, float sep, float* pa, float* pb) {
  const float nn[3] = {-n[0], -n[1], -n[2]};
  const float jA = cvx_jump(A, n), jB = cvx_jump(B, nn);
  const bool sa = jA <= 4e-3f * A.rbound, sb = jB <= 4e-3f * B.rbound;
  if (sa && (!sb || jA <= jB)) {
    cvx_core_support(A, n, pa);
    for (int k = 0; k < 3; k++) pb[k] = pa[k] + sep * n[k];
  } else if (sb) {
    cvx_core_support(B, nn, pb);
    for (int k = 0; k < 3; k++) pa[k] = pb[k] - sep * n[k];
  } else {
    float cA[3], cB[3], sprA, sprB;
    cvx_set_center(A, n, cA, sprA);
    cvx_set_center(B, nn, cB, sprB);
    if (sprA <= sprB) {
      for (int k = 0; k < 3; k++) { pa[k] = cA[k]; pb[k] = cA[k] + sep * n[k]; }
    } else {
      for (int k = 0; k < 3; k++) { pb[k] = cB[k]; pa[k] = cB[k] - sep * n[k]; }
    }
  }
}

__device__ __noinline__ int c_convex(const CShape& A, const CShape& B, float margin, DCon* out) {
  float dir[3] = {B.c[0] - A.c[0], B.c[1] - A.c[1], B.c[2] - A.c[2]};
  if (norm3(dir) < 1e-12f) { dir[0] = 1.f; dir[1] = dir[2] = 0.f; }
  CSV S[4];
  float lam[4], v[3];
  cvx_support(A, B, dir, S[0]);
  int n = 1;
  bool overlap = false;
  for (int k = 0; k < 3; k++) v[k] = S[0].w[k];
  lam[0] = 1.f;
  #pragma unroll 1
  for (int it = 0; it < CVX_ITER; it++) {
    const float vv = dot3(v, v);
    if (vv < CVX_TOL * CVX_TOL) { overlap = true; break; }
    const float nd[3] = {-v[0], -v[1], -v[2]};
    CSV w;
    cvx_support(A, B, nd, w);
    if (vv - dot3(v, w.w) <= CVX_TOL * sqrtf(vv)) break;
    // a support point already in the simplex: v is as close as the simplex
    // gets in this precision (on polytopes FP32 round-off in v can exceed
    // the tolerance and return a vertex again); stop as separated
    bool dup = false;
    for (int i = 0; i < n; i++) {
      const float e[3] = {w.w[0] - S[i].w[0], w.w[1] - S[i].w[1], w.w[2] - S[i].w[2]};
      dup = dup || dot3(e, e) <= 1e-16f;
    }
    if (dup) break;
    S[n++] = w;
    n = cvx_closest(S, n, lam, v);
    if (n == 4) { overlap = true; break; }
  }
  float pa[3] = {0.f, 0.f, 0.f}, pb[3] = {0.f, 0.f, 0.f}, nrm[3], dist;
  if (!overlap) {
    for (int i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) { pa[k] += lam[i] * S[i].a[k]; pb[k] += lam[i] * (S[i].a[k] - S[i].w[k]); }
    float len = norm3(v), h = -len;
    for (int k = 0; k < 3; k++) nrm[k] = -v[k] / len;
    // the separation is -min_n h(n) too (GJK's duality-gap stop leaves the
    // normal only sqrt(tolerance)-accurate on curved shapes)
    CSV sv;
    if (cvx_refine(A, B, nrm, h, sv))
      for (int k = 0; k < 3; k++) { pa[k] = sv.a[k]; pb[k] = sv.a[k] - sv.w[k]; }
    if (-h > 0.f) len = -h;
    cvx_polish(A, B, nrm, len, pa, pb);
    dist = len - A.core - B.core;
  } else {
    float depth;
    if (!cvx_epa(A, B, S, n, depth, nrm, pa, pb)) return 0;
    CSV sv;
    if (cvx_refine(A, B, nrm, depth, sv))
      for (int k = 0; k < 3; k++) { pa[k] = sv.a[k]; pb[k] = sv.a[k] - sv.w[k]; }
    cvx_polish(A, B, nrm, -depth, pa, pb);
    dist = -depth - A.core - B.core;
  }
  if (!(dist < margin)) return 0;
  for (int k = 0; k < 3; k++) {
    pa[k] += A.core * nrm[k];
    pb[k] -= B.core * nrm[k];
    out->pos[k] = 0.5f * (pa[k] + pb[k]);
    out->n[k] = nrm[k];
  }
  out->dist = dist;
  return 1;
}

// Narrowphase of one pair; returns the number of contacts (<= 4), or -1 for a
// type combination without a collider.  CVX = false leaves the GJK / EPA
// collider out (the step kernel instance for models without such pairs, so
// their hot loop carries none of its code).
template <bool CVX>
__device__ __noinline__ int c_collide_pair(int t1, int t2, const float* c1, const float* R1, const float* s1, float rb1, const float* mesh1, int nvert1,
                                              const float* c2, const float* R2, const float* s2, float rb2, const float* mesh2, int nvert2, float margin,
                                              DCon* cs) {
  if (t1 == 0) {
    float pn[3] = {R1[2], R1[5], R1[8]};
    float cd = (c2[0] - c1[0]) * pn[0] + (c2[1] - c1[1]) * pn[1] + (c2[2] - c1[2]) * pn[2];
    if (rb2 > 0 && cd > rb2 + margin) return 0;
    if (t2 == 2) return c_plane_sphere(c1, pn, c2, s2[0], margin, cs);
    if (t2 == 3) return c_plane_capsule(c1, pn, c2, R2, s2, margin, cs);
    if (t2 == 6) return c_plane_box(c1, pn, c2, R2, s2, margin, cs);
    if (t2 == 4 || t2 == 5 || t2 == 7) return c_plane_convex(c1, pn, t2, c2, R2, s2, mesh2, nvert2, margin, cs);
    return -1;
  }
  float v[3] = {c2[0] - c1[0], c2[1] - c1[1], c2[2] - c1[2]};
  if (norm3(v) > rb1 + rb2 + margin) return 0;
  if (t1 == 2 && t2 == 2) return c_sphere_sphere(c1, s1[0], c2, s2[0], margin, cs);
  if (t1 == 2 && t2 == 3) {
    float a0[3], a1[3], q[3];
    for (int k = 0; k < 3; k++) { a0[k] = c2[k] - R2[3 * k + 2] * s2[1]; a1[k] = c2[k] + R2[3 * k + 2] * s2[1]; }
    c_closest_on_segment(a0, a1, c1, q);
    return c_sphere_sphere(c1, s1[0], q, s2[0], margin, cs);
  }
  if (t1 == 3 && t2 == 3) {
    float p1[3], q1[3], p2[3], q2[3], x1[3], x2[3];
    for (int k = 0; k < 3; k++) {
      p1[k] = c1[k] - R1[3 * k + 2] * s1[1]; q1[k] = c1[k] + R1[3 * k + 2] * s1[1];
      p2[k] = c2[k] - R2[3 * k + 2] * s2[1]; q2[k] = c2[k] + R2[3 * k + 2] * s2[1];
    }
    c_segment_segment(p1, q1, p2, q2, x1, x2);
    return c_sphere_sphere(x1, s1[0], x2, s2[0], margin, cs);
  }
  if (t1 == 2 && t2 == 6) return c_sphere_box(c1, s1[0], c2, R2, s2, margin, cs);
  if (t1 == 3 && t2 == 6) return c_capsule_box(c1, R1, s1, c2, R2, s2, margin, cs);
  if (t1 == 6 && t2 == 6) return c_box_box(c1, R1, s1, c2, R2, s2, margin, cs);
  if (CVX && t1 >= 2 && t2 >= 2 && t1 <= 7 && t2 <= 7) {
    const CShape A{t1, nvert1, c1, R1, s1, mesh1, (t1 == 2 || t1 == 3) ? s1[0] : 0.f, rb1};
    const CShape B{t2, nvert2, c2, R2, s2, mesh2, (t2 == 2 || t2 == 3) ? s2[0] : 0.f, rb2};
    return c_convex(A, B, margin, cs);
  }
  return -1;
}

}  // namespace mjbdev
