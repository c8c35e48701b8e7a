// Small batch kernels around the step: masked reset to qpos0
// (reference: mjmlx_batched_reset, src/batched.cpp:1900-1934).
#include <cuda_runtime.h>

#include "devmodel.h"

__global__ void mjb_reset_kernel(const DevModelDesc* models, const int* env_model, const int* qadr, const int* vadr, const float* ftab, const int* mask, int B,
                                 float* qpos, float* qvel, float* warm) {
  int env = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (env >= B || !mask[env]) return;
  const DevModelDesc& m = models[env_model[env]];
  for (int i = lane; i < m.nq; i += 32) qpos[qadr[env] + i] = ftab[m.f_qpos0 + i];
  for (int i = lane; i < m.nv; i += 32) {
    qvel[vadr[env] + i] = 0.f;
    warm[vadr[env] + i] = 0.f;
  }
}

cudaError_t mjb_launch_reset(const DevModelDesc* models, const int* env_model, const int* qadr, const int* vadr, const float* ftab, const int* mask, int B,
                             float* qpos, float* qvel, float* warm, cudaStream_t s) {
  int warps = 8;
  int grid = (B + warps - 1) / warps;
  if (grid < 1) grid = 1;
  mjb_reset_kernel<<<grid, warps * 32, 0, s>>>(models, env_model, qadr, vadr, ftab, mask, B, qpos, qvel, warm);
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
