// Device narrowphase (one lane per candidate pair).  Same contact rules as
// the CPU oracle: plane-sphere 1, plane-capsule 2, plane-box <= 4 deepest
// corners, plane-ellipsoid/cylinder/mesh 1 support point, sphere-sphere,
// sphere-capsule, capsule-capsule, sphere-box, capsule-box 1.  Reference pair
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

// Narrowphase of one pair; returns the number of contacts (<= 4), or -1 for a
// type combination without a collider.
__device__ __noinline__ int c_collide_pair(int t1, int t2, const float* c1, const float* R1, const float* s1, float rb1, const float* c2, const float* R2,
                                              const float* s2, float rb2, const float* mesh2, int nvert2, float margin, DCon* cs) {
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
  return -1;
}

}  // namespace mjbdev
