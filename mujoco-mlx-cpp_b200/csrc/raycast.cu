// Batched ray casting (mj_ray semantics) against the geoms of every env:
// one thread per (env, ray), geom poses from mjb_geom_pose_kernel at the
// envs' current qpos.  Replaces the reference's mjmlx_batched_raycast
// (src/batched.cpp:1729-1893): planes are hit from their +z side only and
// within their half sizes when those are positive; spheres, ellipsoids,
// capsules (cylinder + end spheres), cylinders (side + end discs) and boxes
// (slabs; a ray starting inside returns its exit) are hit; distances are in
// units of the ray vector; -1 means no hit.
#include <cuda_runtime.h>

namespace {

__device__ __forceinline__ float ray_quadratic(float a, float b, float c) {
  // smallest non-negative root of a t^2 + 2 b t + c
  const float disc = b * b - a * c;
  if (disc < 0.f || fabsf(a) < 1e-12f) return -1.f;
  const float sq = sqrtf(disc);
  const float t0 = (-b - sq) / a, t1 = (-b + sq) / a;
  if (t0 >= 0.f) return t0;
  if (t1 >= 0.f) return t1;
  return -1.f;
}

__device__ __forceinline__ float keep_min(float best, float t) { return (t >= 0.f && (best < 0.f || t < best)) ? t : best; }

// Ray p + t v in the geom's local frame.
__device__ float ray_local(int type, const float* s, const float* p, const float* v) {
  switch (type) {
    case 0: {  // plane z = 0, hit from above
      if (v[2] > -1e-12f) return -1.f;
      const float t = -p[2] / v[2];
      if (t < 0.f) return -1.f;
      const float hx = p[0] + t * v[0], hy = p[1] + t * v[1];
      if ((s[0] > 0.f && fabsf(hx) > s[0]) || (s[1] > 0.f && fabsf(hy) > s[1])) return -1.f;
      return t;
    }
    case 2:  // sphere
      return ray_quadratic(v[0] * v[0] + v[1] * v[1] + v[2] * v[2], p[0] * v[0] + p[1] * v[1] + p[2] * v[2],
                           p[0] * p[0] + p[1] * p[1] + p[2] * p[2] - s[0] * s[0]);
    case 4: {  // ellipsoid: unit sphere in scaled coordinates
      const float ps[3] = {p[0] / s[0], p[1] / s[1], p[2] / s[2]}, vs[3] = {v[0] / s[0], v[1] / s[1], v[2] / s[2]};
      return ray_quadratic(vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2], ps[0] * vs[0] + ps[1] * vs[1] + ps[2] * vs[2],
                           ps[0] * ps[0] + ps[1] * ps[1] + ps[2] * ps[2] - 1.f);
    }
    case 3:
    case 5: {  // capsule / cylinder around local z: radius s[0], half length s[1]
      const float r = s[0], h = s[1];
      float best = -1.f;
      const float a = v[0] * v[0] + v[1] * v[1], b = p[0] * v[0] + p[1] * v[1], c = p[0] * p[0] + p[1] * p[1] - r * r;
      const float disc = b * b - a * c;
      if (a > 1e-12f && disc >= 0.f) {
        const float sq = sqrtf(disc);
        const float t0 = (-b - sq) / a, t1 = (-b + sq) / a;
        if (fabsf(p[2] + t0 * v[2]) <= h) best = keep_min(best, t0);
        if (fabsf(p[2] + t1 * v[2]) <= h) best = keep_min(best, t1);
      }
      for (int sgn = -1; sgn <= 1; sgn += 2) {
        if (type == 5) {
          if (fabsf(v[2]) > 1e-12f) {
            const float t = (sgn * h - p[2]) / v[2];
            const float qx = p[0] + t * v[0], qy = p[1] + t * v[1];
            if (t >= 0.f && qx * qx + qy * qy <= r * r) best = keep_min(best, t);
          }
        } else {
          const float pc[3] = {p[0], p[1], p[2] - sgn * h};
          const float a2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2], b2 = pc[0] * v[0] + pc[1] * v[1] + pc[2] * v[2];
          const float c2 = pc[0] * pc[0] + pc[1] * pc[1] + pc[2] * pc[2] - r * r;
          const float d2 = b2 * b2 - a2 * c2;
          if (d2 >= 0.f && a2 > 1e-12f) {
            const float sq = sqrtf(d2);
            const float u0 = (-b2 - sq) / a2, u1 = (-b2 + sq) / a2;
            // only the cap beyond the cylinder end
            if (sgn * (p[2] + u0 * v[2] - sgn * h) >= 0.f) best = keep_min(best, u0);
            if (sgn * (p[2] + u1 * v[2] - sgn * h) >= 0.f) best = keep_min(best, u1);
          }
        }
      }
      return best;
    }
    case 6: {  // box: slabs
      float tn = -1e30f, tf = 1e30f;
      for (int i = 0; i < 3; i++) {
        if (fabsf(v[i]) < 1e-12f) {
          if (fabsf(p[i]) > s[i]) return -1.f;
        } else {
          const float t0 = (-s[i] - p[i]) / v[i], t1 = (s[i] - p[i]) / v[i];
          tn = fmaxf(tn, fminf(t0, t1));
          tf = fminf(tf, fmaxf(t0, t1));
        }
      }
      if (tn > tf || tf < 0.f) return -1.f;
      return tn >= 0.f ? tn : tf;
    }
    default:
      return -1.f;
  }
}

// ginfo[geom_base[model] + g] = {type, size0, size1, size2, include}
__global__ void mjb_ray_kernel(int B, int nray, const int* env_model, const int* geom_base, const int* geom_count, const float* ginfo,
                               const float* gpose, int ng_max, const float* pnt, const float* vec, float* dist, int* geomid) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * nray) return;
  const int env = i / nray;
  const int mdl = env_model[env];
  const int base = geom_base[mdl], ng = geom_count[mdl];
  const float P[3] = {pnt[3 * i], pnt[3 * i + 1], pnt[3 * i + 2]}, V[3] = {vec[3 * i], vec[3 * i + 1], vec[3 * i + 2]};
  float best = -1.f;
  int bg = -1;
  for (int g = 0; g < ng; g++) {
    const float* gi = ginfo + 5 * (base + g);
    if (gi[4] < 0.5f) continue;
    const float* gp = gpose + ((size_t)env * ng_max + g) * 12;
    const float* R = gp + 3;
    const float d[3] = {P[0] - gp[0], P[1] - gp[1], P[2] - gp[2]};
    const float lp[3] = {R[0] * d[0] + R[3] * d[1] + R[6] * d[2], R[1] * d[0] + R[4] * d[1] + R[7] * d[2], R[2] * d[0] + R[5] * d[1] + R[8] * d[2]};
    const float lv[3] = {R[0] * V[0] + R[3] * V[1] + R[6] * V[2], R[1] * V[0] + R[4] * V[1] + R[7] * V[2], R[2] * V[0] + R[5] * V[1] + R[8] * V[2]};
    const float t = ray_local((int)gi[0], gi + 1, lp, lv);
    if (t >= 0.f && (best < 0.f || t < best)) {
      best = t;
      bg = g;
    }
  }
  dist[i] = best;
  geomid[i] = bg;
}

}  // namespace

cudaError_t mjb_launch_ray(int B, int nray, const int* env_model, const int* geom_base, const int* geom_count, const float* ginfo, const float* gpose,
                           int ng_max, const float* pnt, const float* vec, float* dist, int* geomid, cudaStream_t s) {
  const int n = B * nray;
  if (n <= 0) return cudaSuccess;
  mjb_ray_kernel<<<(n + 255) / 256, 256, 0, s>>>(B, nray, env_model, geom_base, geom_count, ginfo, gpose, ng_max, pnt, vec, dist, geomid);
  return cudaGetLastError();
}
