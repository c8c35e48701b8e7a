/* Small double-precision helpers shared by the oracle sources (test infrastructure). */
#ifndef O_UTIL_H
#define O_UTIL_H

#include <math.h>
#include <string.h>

#define O_MINVAL 1e-15

static inline void o_quat_mul(const double a[4], const double b[4], double r[4]) {
  double t[4] = {a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3], a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
                 a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1], a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0]};
  memcpy(r, t, sizeof(t));
}
static inline void o_quat_normalize(double q[4]) {
  double n = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (n < 1e-10) { q[0] = 1; q[1] = q[2] = q[3] = 0; return; }
  q[0] /= n; q[1] /= n; q[2] /= n; q[3] /= n;
}
static inline void o_quat_rot(const double q[4], const double v[3], double r[3]) {
  double w = q[0], x = q[1], y = q[2], z = q[3];
  double t0 = 2 * (x * v[0] + y * v[1] + z * v[2]);
  double t1 = w * w - (x * x + y * y + z * z);
  double o[3] = {t1 * v[0] + t0 * x + 2 * w * (y * v[2] - z * v[1]), t1 * v[1] + t0 * y + 2 * w * (z * v[0] - x * v[2]),
                 t1 * v[2] + t0 * z + 2 * w * (x * v[1] - y * v[0])};
  memcpy(r, o, sizeof(o));
}
static inline void o_quat2mat(const double q[4], double m[9]) {
  double w = q[0], x = q[1], y = q[2], z = q[3];
  m[0] = 1 - 2 * (y * y + z * z); m[1] = 2 * (x * y - w * z); m[2] = 2 * (x * z + w * y);
  m[3] = 2 * (x * y + w * z); m[4] = 1 - 2 * (x * x + z * z); m[5] = 2 * (y * z - w * x);
  m[6] = 2 * (x * z - w * y); m[7] = 2 * (y * z + w * x); m[8] = 1 - 2 * (x * x + y * y);
}
static inline double o_dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void o_cross(const double a[3], const double b[3], double r[3]) {
  double t[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  memcpy(r, t, sizeof(t));
}
static inline double o_norm3(const double a[3]) { return sqrt(o_dot3(a, a)); }
/* world = R * local (R row-major, columns are the frame axes) */
static inline void o_mulmat(const double R[9], const double v[3], double r[3]) {
  double t[3] = {R[0] * v[0] + R[1] * v[1] + R[2] * v[2], R[3] * v[0] + R[4] * v[1] + R[5] * v[2], R[6] * v[0] + R[7] * v[1] + R[8] * v[2]};
  memcpy(r, t, sizeof(t));
}
/* local = R^T * world */
static inline void o_mulmatT(const double R[9], const double v[3], double r[3]) {
  double t[3] = {R[0] * v[0] + R[3] * v[1] + R[6] * v[2], R[1] * v[0] + R[4] * v[1] + R[7] * v[2], R[2] * v[0] + R[5] * v[1] + R[8] * v[2]};
  memcpy(r, t, sizeof(t));
}

/* dense Cholesky in place (lower triangle), returns 0 on success */
static inline int o_chol(double* A, int n) {
  for (int j = 0; j < n; j++) {
    double s = A[j * n + j];
    for (int k = 0; k < j; k++) s -= A[j * n + k] * A[j * n + k];
    if (!(s > 1e-300)) s = 1e-300;
    double dj = sqrt(s);
    A[j * n + j] = dj;
    for (int i = j + 1; i < n; i++) {
      double t = A[i * n + j];
      for (int k = 0; k < j; k++) t -= A[i * n + k] * A[j * n + k];
      A[i * n + j] = t / dj;
    }
  }
  return 0;
}
static inline void o_chol_solve(const double* L, int n, double* x) {
  for (int i = 0; i < n; i++) {
    double s = x[i];
    for (int k = 0; k < i; k++) s -= L[i * n + k] * x[k];
    x[i] = s / L[i * n + i];
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = x[i];
    for (int k = i + 1; k < n; k++) s -= L[k * n + i] * x[k];
    x[i] = s / L[i * n + i];
  }
}

#endif
