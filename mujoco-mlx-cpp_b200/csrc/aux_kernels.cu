// Small batch kernels around the step: masked reset to qpos0
// (reference: mjmlx_batched_reset, src/batched.cpp:1900-1934).
#include <cuda_runtime.h>

#include "devmodel.h"

__global__ void mjb_reset_kernel(const DevModelDesc* models, const int* env_model, const int* qadr, const int* vadr, const float* ftab, const int* mask, int B,
                                 float* qpos, float* qvel, float* warm, int* sens_valid) {
  int env = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (env >= B || !mask[env]) return;
  const DevModelDesc& m = models[env_model[env]];
  // accelerometers restart without a previous velocity (sensor.cpp sensor_mark_reset)
  if (sens_valid && lane == 0) sens_valid[env] = 0;
  for (int i = lane; i < m.nq; i += 32) qpos[qadr[env] + i] = ftab[m.f_qpos0 + i];
  for (int i = lane; i < m.nv; i += 32) {
    qvel[vadr[env] + i] = 0.f;
    warm[vadr[env] + i] = 0.f;
  }
}

cudaError_t mjb_launch_reset(const DevModelDesc* models, const int* env_model, const int* qadr, const int* vadr, const float* ftab, const int* mask, int B,
                             float* qpos, float* qvel, float* warm, int* sens_valid, cudaStream_t s) {
  int warps = 8;
  int grid = (B + warps - 1) / warps;
  if (grid < 1) grid = 1;
  mjb_reset_kernel<<<grid, warps * 32, 0, s>>>(models, env_model, qadr, vadr, ftab, mask, B, qpos, qvel, warm, sens_valid);
  return cudaGetLastError();
}

// out = a - b elementwise (training targets of the learned warm start).
__global__ void mjb_sub_kernel(int n, const float* a, const float* b, float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] - b[i];
}

cudaError_t mjb_sub(int n, const float* a, const float* b, float* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  mjb_sub_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, a, b, out);
  return cudaGetLastError();
}

// Packed read-back row per env (uniform batch): [qpos (nq), qvel (nv),
// |force part of cfrc_ext| of each selected body, sum qfrc_actuator^2 and
// sum |qfrc_actuator| over dofs [dof_lo, dof_lo + ndof)] (reference:
// mjmlx_batched_get_pack, src/batched.cpp:1675-1727).  One warp per env.
__global__ void mjb_pack_kernel(int B, int nq, int nv, int nbody, const float* qpos, const float* qvel, const float* cfrc, const float* qfa,
                                const int* bodies, int nsel, int dof_lo, int ndof, int stride, float* out) {
  const int env = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (env >= B) return;
  float* row = out + (size_t)env * stride;
  for (int i = lane; i < nq; i += 32) row[i] = qpos[(size_t)env * nq + i];
  for (int i = lane; i < nv; i += 32) row[nq + i] = qvel[(size_t)env * nv + i];
  for (int k = lane; k < nsel; k += 32) {
    const float* f = cfrc + ((size_t)env * nbody + bodies[k]) * 6 + 3;
    row[nq + nv + k] = sqrtf(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
  }
  float s2 = 0.f, s1 = 0.f;
  for (int d = lane; d < ndof; d += 32) {
    const float v = qfa[(size_t)env * nv + dof_lo + d];
    s2 += v * v;
    s1 += fabsf(v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
  if (lane == 0) {
    row[nq + nv + nsel] = s2;
    row[nq + nv + nsel + 1] = s1;
  }
}

cudaError_t mjb_launch_pack(int B, int nq, int nv, int nbody, const float* qpos, const float* qvel, const float* cfrc, const float* qfa, const int* bodies,
                            int nsel, int dof_lo, int ndof, int stride, float* out, cudaStream_t s) {
  if (B <= 0) return cudaSuccess;
  mjb_pack_kernel<<<(B + 7) / 8, 256, 0, s>>>(B, nq, nv, nbody, qpos, qvel, cfrc, qfa, bodies, nsel, dof_lo, ndof, stride, out);
  return cudaGetLastError();
}
