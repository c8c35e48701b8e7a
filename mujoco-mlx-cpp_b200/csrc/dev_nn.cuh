// Learned Newton warm start fused into the step kernel (per-env models,
// lockstep CTAs; no counterpart in the reference).
//
// After the constraint build of every substep, each warp writes its env's
// feature row (the state of the substep, its unconstrained acceleration, the
// previous converged acceleration, the controls and the first contacts) as a
// normalised bf16 row into an idle part of its workspace (the Hessian slot,
// which Newton fills only later).  The warps of the CTA then evaluate the
// 4-layer MLP on those rows together: every layer is a [16 x K] x [K x N]
// product on mma.sync m16n8k16 tensor-core tiles (bf16 operands, fp32
// accumulation), each warp owning N / 8 / W output tiles for all rows (W = 8
// or 16 warps per CTA), with
// the weights read straight from L2 as 16-byte fragments.  Rows past the
// CTA's W envs repeat its rows and are discarded.  The output layer writes
// qacc_prev + mean + std * y into solver vector slot 7 of each env, which the
// Newton solver offers as a warm-start candidate.
//
// Operand layout: within each 32-wide K chunk, lane t of a quad loads the 8
// consecutive bf16 at k0 + 8 t of its A rows and of its B row in one 16-byte
// access; the chunk's two MMAs take them as K positions {2t, 2t+1, 2t+8,
// 2t+9} (first 4) and the same of the second MMA (last 4).  A and B use the
// same K permutation, so the sum over K is unchanged.
#pragma once
#include <cuda_bf16.h>

#include "dev_stages.cuh"

namespace mjbdev {

// Raw feature j of the env (the fused warm start's input layout):
// qpos[qskip:nq], qvel, qacc_smooth, previous converged qacc, ctrl, then the
// normal and distance of the first MJB_FEAT_CONTACTS contacts (zero padded).
__device__ __forceinline__ int nn_feature_count(const DevModelDesc& m, int qskip) { return m.nq - qskip + 3 * m.nv + m.nu + 4 * MJB_FEAT_CONTACTS; }

__device__ __forceinline__ float nn_feature(const DevModelDesc& m, const float* ws, int qskip, int ncon, int j) {
  const int nqf = m.nq - qskip, nv = m.nv;
  if (j < nqf) return ws[m.w_qpos + qskip + j];
  j -= nqf;
  if (j < nv) return ws[m.w_qvel + j];
  j -= nv;
  if (j < nv) return ws[m.w_qas + j];
  j -= nv;
  if (j < nv) return ws[m.w_xwarm + j];
  j -= nv;
  if (j < m.nu) return ws[m.w_ctrl + j];
  j -= m.nu;
  const int c = j >> 2, q = j & 3;
  if (c >= ncon) return 0.f;
  const float* con = ws + m.w_con + c * MJB_CONTACT_FLOATS;
  return q < 3 ? con[3 + q] : con[12];
}

// Activation buffer b (0 or 1, 256 bf16 each) of the env whose workspace is ws.
__device__ __forceinline__ __nv_bfloat16* nn_act(const DevModelDesc& m, float* ws, int b) { return reinterpret_cast<__nv_bfloat16*>(ws + m.w_H) + 256 * b; }

// Feature row of one env: raw values to raw_out (training pairs, may be
// null) and the normalised bf16 row, zero padded to the first layer's width,
// into activation buffer 0 (when P.nn_w[0] is set).  valid = false zeroes the
// row (envs past the batch in the last CTA).
__device__ __noinline__ void d_nn_features(const Env& E, const StepParams& P, int ncon, bool valid, float* raw_out) {
  const DevModelDesc& m = *E.md;
  const int F = P.nn_in_raw, K0 = P.nn_cols[0];
  __nv_bfloat16* row = P.nn_w[0] ? nn_act(m, E.ws, 0) : nullptr;
#pragma unroll 1
  for (int j = E.lane; j < (row ? K0 : F); j += 32) {
    const float f = valid && j < F ? nn_feature(m, E.ws, P.feat_qskip, ncon, j) : 0.f;
    if (raw_out && valid && j < F) raw_out[j] = f;
    if (row) row[j] = __float2bfloat16_rn(j < F ? (f - __ldg(P.nn_in_mean + j)) * __ldg(P.nn_in_istd + j) : 0.f);
  }
  __syncwarp();
}

// (not volatile: the compiler may schedule the MMAs and weight loads freely)
__device__ __forceinline__ void mma_16816(float* c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint4 ldg_v4(const uint16_t* p) { return __ldg(reinterpret_cast<const uint4*>(p)); }

__device__ __forceinline__ float nn_gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }

// One layer for the CTA: rows 0..15 (row r = env of warp r % W), input
// buffer l & 1, output buffer (l + 1) & 1 (hidden layers) or the prediction
// (output layer).  TPW = output tiles of 8 columns per warp (32 / W).
template <int TPW>
__device__ __forceinline__ void nn_layer(const StepParams& P, const DevModelDesc& m, float* ws0, int stride, int W, int warp, int lane, int l) {
  const int K = P.nn_cols[l];
  const bool last = l == 3;
  const int ntile = last ? (P.nn_nout + 7) >> 3 : P.nn_rows[l] >> 3;
  const int g = lane >> 2, t = lane & 3;
  const int rg = g % W, rh = (g + 8) % W;
  const __nv_bfloat16* ag = nn_act(m, ws0 + (size_t)rg * stride, l & 1) + 8 * t;
  const __nv_bfloat16* ah = nn_act(m, ws0 + (size_t)rh * stride, l & 1) + 8 * t;
  const uint16_t* wl = P.nn_w[l] + (size_t)g * K + 8 * t;
  float acc[TPW][4];
  bool on[TPW];
  const uint16_t* wt[TPW];
#pragma unroll
  for (int i = 0; i < TPW; i++) {
    acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
    on[i] = warp + i * W < ntile;
    wt[i] = wl + (size_t)(warp + i * W) * 8 * K;
  }
  // each chunk's weight fragments are loaded one chunk ahead of its MMAs, all
  // of the warp's tiles together; tiles past ntile load nothing
  uint4 b0[TPW];
#pragma unroll
  for (int i = 0; i < TPW; i++) b0[i] = on[i] ? ldg_v4(wt[i]) : make_uint4(0, 0, 0, 0);
#pragma unroll 1
  for (int k0 = 0; k0 < K; k0 += 32) {
    uint4 b1[TPW];
#pragma unroll
    for (int i = 0; i < TPW; i++) b1[i] = on[i] && k0 + 32 < K ? ldg_v4(wt[i] + k0 + 32) : make_uint4(0, 0, 0, 0);
    const uint4 a = *reinterpret_cast<const uint4*>(ag + k0);
    const uint4 h = *reinterpret_cast<const uint4*>(ah + k0);
#pragma unroll
    for (int i = 0; i < TPW; i++) {
      if (on[i]) {
        mma_16816(acc[i], a.x, h.x, a.y, h.y, b0[i].x, b0[i].y);
        mma_16816(acc[i], a.z, h.z, a.w, h.w, b0[i].z, b0[i].w);
      }
      b0[i] = b1[i];
    }
  }
  const float* bias = P.nn_b[l];
#pragma unroll
  for (int i = 0; i < TPW; i++) {
    const int tile = warp + i * W;
    if (tile >= ntile) continue;
    const int n = tile * 8 + 2 * t;
    const float b0 = __ldg(bias + n), b1 = __ldg(bias + n + 1);
    const float v[4] = {acc[i][0] + b0, acc[i][1] + b1, acc[i][2] + b0, acc[i][3] + b1};
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const int r = g + 8 * half;
      if (r >= W) continue;
      float* wsr = ws0 + (size_t)r * stride;
      if (!last) {
        const __nv_bfloat162 o = __floats2bfloat162_rn(nn_gelu(v[2 * half]), nn_gelu(v[2 * half + 1]));
        *reinterpret_cast<__nv_bfloat162*>(nn_act(m, wsr, (l + 1) & 1) + n) = o;
      } else {
        float* pred = wsr + m.w_vec + 7 * m.nv;
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const int col = n + c;
          if (col < P.nn_nout) pred[col] = wsr[m.w_xwarm + col] + __ldg(P.nn_out_mean + col) + __ldg(P.nn_out_std + col) * v[2 * half + c];
        }
      }
    }
  }
}

// The MLP for the CTA's envs after every warp has written its feature row
// (d_nn_features); called by all threads of the CTA (it holds block
// barriers).  ws0: workspace of warp 0; W: warps per CTA (8 or 16).
__device__ __noinline__ void d_nn_infer(const StepParams& P, const DevModelDesc& m, float* ws0, int W, int warp, int lane) {
  __syncthreads();
#pragma unroll 1
  for (int l = 0; l < 4; l++) {
    if (W == 16) nn_layer<2>(P, m, ws0, P.ws_stride, W, warp, lane, l);
    else nn_layer<4>(P, m, ws0, P.ws_stride, W, warp, lane, l);
    __syncthreads();
  }
}

}  // namespace mjbdev
