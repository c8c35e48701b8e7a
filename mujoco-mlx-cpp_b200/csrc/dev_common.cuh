// Device helpers: warp collectives and small-vector math (float).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "devmodel.h"

#define FULL_MASK 0xffffffffu

namespace mjbdev {

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(FULL_MASK, v, o));
  return v;
}
__device__ __forceinline__ int warp_sum_int(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
  return v;
}
// inclusive scan over lanes
__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(FULL_MASK, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

__device__ __forceinline__ void qmul(const float a[4], const float b[4], float r[4]) {
  float t0 = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  float t1 = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  float t2 = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  float t3 = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
  r[0] = t0; r[1] = t1; r[2] = t2; r[3] = t3;
}
__device__ __forceinline__ void qnormalize(float q[4]) {
  float n = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (n < 1e-10f) { q[0] = 1; q[1] = q[2] = q[3] = 0; return; }
  float in = 1.0f / n;
  q[0] *= in; q[1] *= in; q[2] *= in; q[3] *= in;
}
__device__ __forceinline__ void qrot(const float q[4], const float v[3], float r[3]) {
  float w = q[0], x = q[1], y = q[2], z = q[3];
  float t0 = 2.f * (x * v[0] + y * v[1] + z * v[2]);
  float t1 = w * w - (x * x + y * y + z * z);
  float o0 = t1 * v[0] + t0 * x + 2.f * w * (y * v[2] - z * v[1]);
  float o1 = t1 * v[1] + t0 * y + 2.f * w * (z * v[0] - x * v[2]);
  float o2 = t1 * v[2] + t0 * z + 2.f * w * (x * v[1] - y * v[0]);
  r[0] = o0; r[1] = o1; r[2] = o2;
}
__device__ __forceinline__ void q2mat(const float q[4], float m[9]) {
  float w = q[0], x = q[1], y = q[2], z = q[3];
  m[0] = 1 - 2 * (y * y + z * z); m[1] = 2 * (x * y - w * z); m[2] = 2 * (x * z + w * y);
  m[3] = 2 * (x * y + w * z); m[4] = 1 - 2 * (x * x + z * z); m[5] = 2 * (y * z - w * x);
  m[6] = 2 * (x * z - w * y); m[7] = 2 * (y * z + w * x); m[8] = 1 - 2 * (x * x + y * y);
}
__device__ __forceinline__ float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ void cross3(const float a[3], const float b[3], float r[3]) {
  float t0 = a[1] * b[2] - a[2] * b[1], t1 = a[2] * b[0] - a[0] * b[2], t2 = a[0] * b[1] - a[1] * b[0];
  r[0] = t0; r[1] = t1; r[2] = t2;
}
__device__ __forceinline__ float norm3(const float a[3]) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ void mulmat(const float* R, const float v[3], float r[3]) {
  float t0 = R[0] * v[0] + R[1] * v[1] + R[2] * v[2];
  float t1 = R[3] * v[0] + R[4] * v[1] + R[5] * v[2];
  float t2 = R[6] * v[0] + R[7] * v[1] + R[8] * v[2];
  r[0] = t0; r[1] = t1; r[2] = t2;
}
__device__ __forceinline__ void mulmatT(const float* R, const float v[3], float r[3]) {
  float t0 = R[0] * v[0] + R[3] * v[1] + R[6] * v[2];
  float t1 = R[1] * v[0] + R[4] * v[1] + R[7] * v[2];
  float t2 = R[2] * v[0] + R[5] * v[1] + R[8] * v[2];
  r[0] = t0; r[1] = t1; r[2] = t2;
}
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }

// One constraint row of the structure-of-arrays row table: field f of row r
// lives at base[f * ne] with base = efc + r, so lanes that walk consecutive
// rows touch consecutive words (no shared-memory bank conflicts).
struct EfcRef {
  float* base;
  int ne;
  __device__ __forceinline__ float& operator[](int f) const { return base[f * ne]; }
};

// Dot products with four independent accumulators (instruction-level
// parallelism instead of one long dependent FMA chain).
__device__ __forceinline__ float dot_c(const float* a, const float* b, int n) {
  float s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  int k = 0;
#pragma unroll 1
  for (; k + 3 < n; k += 4) {
    s0 += a[k] * b[k];
    s1 += a[k + 1] * b[k + 1];
    s2 += a[k + 2] * b[k + 2];
    s3 += a[k + 3] * b[k + 3];
  }
#pragma unroll 1
  for (; k < n; k++) s0 += a[k] * b[k];
  return (s0 + s1) + (s2 + s3);
}
// sum_k a[k * stride] * b[k]
__device__ __forceinline__ float dot_s(const float* a, int stride, const float* b, int n) {
  float s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  int k = 0;
#pragma unroll 1
  for (; k + 3 < n; k += 4) {
    s0 += a[k * stride] * b[k];
    s1 += a[(k + 1) * stride] * b[k + 1];
    s2 += a[(k + 2) * stride] * b[k + 2];
    s3 += a[(k + 3) * stride] * b[k + 3];
  }
#pragma unroll 1
  for (; k < n; k++) s0 += a[k * stride] * b[k];
  return (s0 + s1) + (s2 + s3);
}

// read-only model table access (L1/L2 cached, tables are shared by every env)
// t may be the shared-memory copy of the int table or the global one: a
// generic load serves both
__device__ __forceinline__ int ldi(const int* t, int i) { return t[i]; }
__device__ __forceinline__ float ldf(const float* t, int i) { return __ldg(t + i); }

}  // namespace mjbdev
