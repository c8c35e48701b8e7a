// Warp-cooperative stages of the physics step, one warp per env, all
// intermediate state in the warp's shared-memory workspace.
//   d_kinematics  <- kinematics.hpp:75-183 (bodies processed level by level,
//                    one lane per body of the level)
//   d_collide     <- collision.hpp:235-501 (one lane per candidate pair;
//                    contacts compacted in pair order with a warp scan)
//   d_com/d_crb   <- forward.hpp:143-279
//   d_rne         <- forward.hpp:281-397
//   d_forces      <- forward.hpp:399-469
#pragma once
#include "dev_collide.cuh"
#include "tendon_wrap.h"
#include "step_params.h"

namespace mjbdev {

// The lane index, read from the thread index wherever E.lane is used
// (it converts to int), so the rest of the context can live in one
// per-warp shared-memory slot.
struct LaneId {
  __device__ __forceinline__ operator int() const { return (int)(threadIdx.x & 31u); }
};

// Per-env context of a warp.  The step kernels keep it in the warp's
// shared-memory slot after the model descriptor copy, and the stage
// functions take it by reference, so reading a field is a shared-memory
// load rather than a stack load.  Status bits are set with atomicOr
// (env_status), which is safe from any subset of the warp's lanes.
struct Env {
  const DevModelDesc* md;  // shared-memory copy
  const int* it;
  const float* ft;
  float* ws;
  int env;
  int status;
  LaneId lane;
};

__device__ __forceinline__ void env_status(Env& E, int bits) { atomicOr(&E.status, bits); }
static_assert(sizeof(Env) <= 4 * MJB_ENV_SLOT_WORDS, "env context exceeds its shared-memory slot");

__device__ __forceinline__ float msc(const StepParams& P, const Env& E, int b) {
  return P.rand_mass ? P.rand_mass[P.env_badr[E.env] + b] : 1.f;
}

__device__ __noinline__ void d_kinematics(Env& E) {
  const DevModelDesc& m = *E.md;
  const int* it = E.it;
  const float* ft = E.ft;
  float* ws = E.ws;
  const float* qpos = ws + m.w_qpos;
  float* xpos = ws + m.w_xpos;
  float* xquat = ws + m.w_xquat;
  float* xmat = ws + m.w_xmat;
  float* xipos = ws + m.w_xipos;
  float* xanchor = ws + m.w_xanchor;
  float* xaxis = ws + m.w_xaxis;
  if (E.lane == 0) {
    xpos[0] = xpos[1] = xpos[2] = 0;
    xquat[0] = 1; xquat[1] = xquat[2] = xquat[3] = 0;
  }
  __syncwarp();
  #pragma unroll 1
  for (int l = 1; l < m.nlevel; l++) {
    int s = ldi(it, m.i_level_start + l), e = ldi(it, m.i_level_start + l + 1);
    #pragma unroll 1
    for (int k = s + E.lane; k < e; k += 32) {
      int b = ldi(it, m.i_level_body + k);
      int p = ldi(it, m.i_body_parentid + b);
      float pq[4] = {xquat[4 * p], xquat[4 * p + 1], xquat[4 * p + 2], xquat[4 * p + 3]};
      float lp[3] = {ldf(ft, m.f_body_pos + 3 * b), ldf(ft, m.f_body_pos + 3 * b + 1), ldf(ft, m.f_body_pos + 3 * b + 2)};
      float lq[4] = {ldf(ft, m.f_body_quat + 4 * b), ldf(ft, m.f_body_quat + 4 * b + 1), ldf(ft, m.f_body_quat + 4 * b + 2), ldf(ft, m.f_body_quat + 4 * b + 3)};
      float pos[3], quat[4], r[3];
      qrot(pq, lp, r);
      for (int c = 0; c < 3; c++) pos[c] = xpos[3 * p + c] + r[c];
      qmul(pq, lq, quat);
      int ja = ldi(it, m.i_body_jntadr + b), jn = ldi(it, m.i_body_jntnum + b);
      #pragma unroll 1
      for (int j = ja; j >= 0 && j < ja + jn; j++) {
        int t = ldi(it, m.i_jnt_type + j);
        int qa = ldi(it, m.i_jnt_qposadr + j);
        float* an = xanchor + 3 * j;
        float* ax = xaxis + 3 * j;
        if (t == 0) {
          for (int c = 0; c < 3; c++) pos[c] = qpos[qa + c];
          for (int c = 0; c < 4; c++) quat[c] = qpos[qa + 3 + c];
          qnormalize(quat);
          for (int c = 0; c < 3; c++) an[c] = pos[c];
          ax[0] = 0; ax[1] = 0; ax[2] = 1;
          continue;
        }
        float jp[3] = {ldf(ft, m.f_jnt_pos + 3 * j), ldf(ft, m.f_jnt_pos + 3 * j + 1), ldf(ft, m.f_jnt_pos + 3 * j + 2)};
        float ja3[3] = {ldf(ft, m.f_jnt_axis + 3 * j), ldf(ft, m.f_jnt_axis + 3 * j + 1), ldf(ft, m.f_jnt_axis + 3 * j + 2)};
        float rj[3], axw[3];
        qrot(quat, jp, rj);
        for (int c = 0; c < 3; c++) an[c] = pos[c] + rj[c];
        qrot(quat, ja3, axw);
        for (int c = 0; c < 3; c++) ax[c] = axw[c];
        if (t == 3 || t == 1) {
          float ql[4];
          if (t == 3) {
            float ang = qpos[qa] - ldf(ft, m.f_qpos0 + qa);
            float sn, cs;
            sincosf(0.5f * ang, &sn, &cs);
            ql[0] = cs; ql[1] = ja3[0] * sn; ql[2] = ja3[1] * sn; ql[3] = ja3[2] * sn;
          } else {
            for (int c = 0; c < 4; c++) ql[c] = qpos[qa + c];
            qnormalize(ql);
          }
          qmul(quat, ql, quat);
          qrot(quat, jp, rj);
          for (int c = 0; c < 3; c++) pos[c] = an[c] - rj[c];
        } else {
          float dist = qpos[qa] - ldf(ft, m.f_qpos0 + qa);
          for (int c = 0; c < 3; c++) pos[c] += axw[c] * dist;
        }
      }
      qnormalize(quat);
      for (int c = 0; c < 3; c++) xpos[3 * b + c] = pos[c];
      for (int c = 0; c < 4; c++) xquat[4 * b + c] = quat[c];
    }
    __syncwarp();
  }
  #pragma unroll 1
  for (int b = E.lane; b < m.nbody; b += 32) {
    float q[4] = {xquat[4 * b], xquat[4 * b + 1], xquat[4 * b + 2], xquat[4 * b + 3]};
    q2mat(q, xmat + 9 * b);
    float ip[3] = {ldf(ft, m.f_body_ipos + 3 * b), ldf(ft, m.f_body_ipos + 3 * b + 1), ldf(ft, m.f_body_ipos + 3 * b + 2)}, r[3];
    qrot(q, ip, r);
    for (int c = 0; c < 3; c++) xipos[3 * b + c] = xpos[3 * b + c] + r[c];
  }
  float* gxpos = ws + m.w_gxpos;
  float* gxmat = ws + m.w_gxmat;
  #pragma unroll 1
  for (int g = E.lane; g < m.ngeom; g += 32) {
    int b = ldi(it, m.i_geom_bodyid + g);
    float q[4] = {xquat[4 * b], xquat[4 * b + 1], xquat[4 * b + 2], xquat[4 * b + 3]};
    float gp[3] = {ldf(ft, m.f_geom_pos + 3 * g), ldf(ft, m.f_geom_pos + 3 * g + 1), ldf(ft, m.f_geom_pos + 3 * g + 2)}, r[3];
    float gq[4] = {ldf(ft, m.f_geom_quat + 4 * g), ldf(ft, m.f_geom_quat + 4 * g + 1), ldf(ft, m.f_geom_quat + 4 * g + 2), ldf(ft, m.f_geom_quat + 4 * g + 3)}, cq[4];
    qrot(q, gp, r);
    for (int c = 0; c < 3; c++) gxpos[3 * g + c] = xpos[3 * b + c] + r[c];
    qmul(q, gq, cq);
    q2mat(cq, gxmat + 9 * g);
  }
  __syncwarp();
}

// Broadphase + narrowphase; contacts in pair order.  Returns ncon.
template <bool CVX>
__device__ __noinline__ int d_collide(Env& E) {
  const DevModelDesc& m = *E.md;
  const int* it = E.it;
  const float* ft = E.ft;
  float* ws = E.ws;
  const float* gxpos = ws + m.w_gxpos;
  const float* gxmat = ws + m.w_gxmat;
  float* con = ws + m.w_con;
  int ncon = 0;
  if (m.disableflags & ((1 << 0) | (1 << 4))) return 0;
  #pragma unroll 1
  for (int base = 0; base < m.npair; base += 32) {
    int p = base + E.lane;
    DCon cs[4];
    int n = 0;
    bool unsup = false;
    if (p < m.npair) {
      int g1 = ldi(it, m.i_pair + 6 * p), g2 = ldi(it, m.i_pair + 6 * p + 1);
      int t1 = ldi(it, m.i_geom_type + g1), t2 = ldi(it, m.i_geom_type + g2);
      float margin = ldf(ft, m.f_pair + 16 * p);
      float s1[3] = {ldf(ft, m.f_geom_size + 3 * g1), ldf(ft, m.f_geom_size + 3 * g1 + 1), ldf(ft, m.f_geom_size + 3 * g1 + 2)};
      float s2[3] = {ldf(ft, m.f_geom_size + 3 * g2), ldf(ft, m.f_geom_size + 3 * g2 + 1), ldf(ft, m.f_geom_size + 3 * g2 + 2)};
      const float *mesh1 = nullptr, *mesh2 = nullptr;
      int nvert1 = 0, nvert2 = 0;
      if (t1 == 7) {
        int md = ldi(it, m.i_geom_dataid + g1);
        mesh1 = ft + m.f_mesh_vert + 3 * ldi(it, m.i_mesh + 2 * md);
        nvert1 = ldi(it, m.i_mesh + 2 * md + 1);
      }
      if (t2 == 7) {
        int md = ldi(it, m.i_geom_dataid + g2);
        mesh2 = ft + m.f_mesh_vert + 3 * ldi(it, m.i_mesh + 2 * md);
        nvert2 = ldi(it, m.i_mesh + 2 * md + 1);
      }
      n = c_collide_pair<CVX>(t1, t2, gxpos + 3 * g1, gxmat + 9 * g1, s1, ldf(ft, m.f_geom_rbound + g1), mesh1, nvert1, gxpos + 3 * g2, gxmat + 9 * g2,
                         s2, ldf(ft, m.f_geom_rbound + g2), mesh2, nvert2, margin, cs);
      if (n < 0) { unsup = true; n = 0; }
    }
    if (__any_sync(FULL_MASK, unsup)) env_status(E, MJB_STATUS_UNSUPPORTED_PAIR);
    int incl = warp_incl_scan(n, E.lane);
    int total = __shfl_sync(FULL_MASK, incl, 31);
    int off = ncon + incl - n;
    #pragma unroll 1
    for (int i = 0; i < n; i++) {
      int idx = off + i;
      if (idx >= m.ncon_max) break;
      float* c = con + MJB_CONTACT_FLOATS * idx;
      for (int k = 0; k < 3; k++) c[k] = cs[i].pos[k];
      c_make_frame(cs[i].n, c + 3);
      c[12] = cs[i].dist;
      c[13] = (float)p;
      c[14] = (float)ldi(it, m.i_pair + 6 * p + 4);
      c[15] = ldf(ft, m.f_pair + 16 * p + 1);
    }
    ncon += total;
  }
  if (ncon > m.ncon_max) {
    env_status(E, MJB_STATUS_CONTACT_OVERFLOW);
    ncon = m.ncon_max;
  }
  __syncwarp();
  return ncon;
}

// subtree COM, cinert (about the root's subtree COM), cdof
__device__ __noinline__ void d_com(Env& E, const StepParams& P) {
  const DevModelDesc& m = *E.md;
  const int* it = E.it;
  const float* ft = E.ft;
  float* ws = E.ws;
  float* tmp = ws + m.w_tmp;  // 4 per body: mass, mass*xipos
  float* xipos = ws + m.w_xipos;
  const float* xquat = ws + m.w_xquat;
  float* scom = ws + m.w_scom;
  if (P.rand_com) {
    // per-env COM offset in the body frame (reference: forward.hpp:110-115)
    const float* cd = P.rand_com + 3 * P.env_badr[E.env];
    const float* xmat = ws + m.w_xmat;
    #pragma unroll 1
    for (int b = 1 + E.lane; b < m.nbody; b += 32) {
      const float d[3] = {cd[3 * b], cd[3 * b + 1], cd[3 * b + 2]};
      float w[3];
      mulmat(xmat + 9 * b, d, w);
      for (int k = 0; k < 3; k++) xipos[3 * b + k] += w[k];
    }
    __syncwarp();
  }
  #pragma unroll 1
  for (int b = E.lane; b < m.nbody; b += 32) {
    float mb = ldf(ft, m.f_body_mass + b) * msc(P, E, b);
    tmp[4 * b] = mb;
    for (int c = 0; c < 3; c++) tmp[4 * b + 1 + c] = mb * xipos[3 * b + c];
  }
  __syncwarp();
  for (int l = m.nlevel - 2; l >= 0; l--) {
    int s = ldi(it, m.i_level_start + l), e = ldi(it, m.i_level_start + l + 1);
    #pragma unroll 1
    for (int k = s + E.lane; k < e; k += 32) {
      int b = ldi(it, m.i_level_body + k);
      int c0 = ldi(it, m.i_child_start + b), c1 = ldi(it, m.i_child_start + b + 1);
      float a[4] = {tmp[4 * b], tmp[4 * b + 1], tmp[4 * b + 2], tmp[4 * b + 3]};
      #pragma unroll 1
      for (int ci = c0; ci < c1; ci++) {
        int c = ldi(it, m.i_child_list + ci);
        for (int q = 0; q < 4; q++) a[q] += tmp[4 * c + q];
      }
      for (int q = 0; q < 4; q++) tmp[4 * b + q] = a[q];
    }
    __syncwarp();
  }
  #pragma unroll 1
  for (int b = E.lane; b < m.nbody; b += 32) {
    float mass = tmp[4 * b];
    for (int c = 0; c < 3; c++) scom[3 * b + c] = mass > 1e-8f ? tmp[4 * b + 1 + c] / mass : xipos[3 * b + c];
  }
  __syncwarp();
  float* cinert = ws + m.w_cinert;
  #pragma unroll 1
  for (int b = E.lane; b < m.nbody; b += 32) {
    float* ci = cinert + 10 * b;
    if (b == 0) {
      for (int k = 0; k < 10; k++) ci[k] = 0;
      continue;
    }
    float s = msc(P, E, b);
    float mb = ldf(ft, m.f_body_mass + b) * s;
    float q[4] = {xquat[4 * b], xquat[4 * b + 1], xquat[4 * b + 2], xquat[4 * b + 3]};
    float iq[4] = {ldf(ft, m.f_body_iquat + 4 * b), ldf(ft, m.f_body_iquat + 4 * b + 1), ldf(ft, m.f_body_iquat + 4 * b + 2), ldf(ft, m.f_body_iquat + 4 * b + 3)};
    float cq[4], R[9];
    qmul(q, iq, cq);
    q2mat(cq, R);
    float I0 = ldf(ft, m.f_body_inertia + 3 * b) * s, I1 = ldf(ft, m.f_body_inertia + 3 * b + 1) * s, I2 = ldf(ft, m.f_body_inertia + 3 * b + 2) * s;
    float Ig[9];
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) Ig[r * 3 + c] = R[r * 3] * I0 * R[c * 3] + R[r * 3 + 1] * I1 * R[c * 3 + 1] + R[r * 3 + 2] * I2 * R[c * 3 + 2];
    int root = ldi(it, m.i_body_rootid + b);
    float off[3] = {xipos[3 * b] - scom[3 * root], xipos[3 * b + 1] - scom[3 * root + 1], xipos[3 * b + 2] - scom[3 * root + 2]};
    float d2 = dot3(off, off);
    ci[0] = Ig[0] + mb * (d2 - off[0] * off[0]);
    ci[1] = Ig[4] + mb * (d2 - off[1] * off[1]);
    ci[2] = Ig[8] + mb * (d2 - off[2] * off[2]);
    ci[3] = Ig[1] - mb * off[0] * off[1];
    ci[4] = Ig[2] - mb * off[0] * off[2];
    ci[5] = Ig[5] - mb * off[1] * off[2];
    ci[6] = mb * off[0]; ci[7] = mb * off[1]; ci[8] = mb * off[2];
    ci[9] = mb;
  }
  float* cdof = ws + m.w_cdof;
  const float* xmat = ws + m.w_xmat;
  const float* xanchor = ws + m.w_xanchor;
  const float* xaxis = ws + m.w_xaxis;
  #pragma unroll 1
  for (int i = E.lane; i < m.nv; i += 32) {
    int b = ldi(it, m.i_dof_bodyid + i), j = ldi(it, m.i_dof_jntid + i), t = ldi(it, m.i_jnt_type + j);
    int sub = i - ldi(it, m.i_jnt_dofadr + j);
    float* c = cdof + 6 * i;
    int root = ldi(it, m.i_body_rootid + b);
    float ax[3];
    bool rot = true;
    if (t == 3) { ax[0] = xaxis[3 * j]; ax[1] = xaxis[3 * j + 1]; ax[2] = xaxis[3 * j + 2]; }
    else if (t == 2) { rot = false; ax[0] = xaxis[3 * j]; ax[1] = xaxis[3 * j + 1]; ax[2] = xaxis[3 * j + 2]; }
    else if (t == 0 && sub < 3) { rot = false; ax[0] = ax[1] = ax[2] = 0; ax[sub] = 1; }
    else {
      int col = (t == 0) ? sub - 3 : sub;
      for (int k = 0; k < 3; k++) ax[k] = xmat[9 * b + 3 * k + col];
    }
    if (rot) {
      float off[3] = {scom[3 * root] - xanchor[3 * j], scom[3 * root + 1] - xanchor[3 * j + 1], scom[3 * root + 2] - xanchor[3 * j + 2]};
      c[0] = ax[0]; c[1] = ax[1]; c[2] = ax[2];
      cross3(ax, off, c + 3);
    } else {
      c[0] = c[1] = c[2] = 0;
      c[3] = ax[0]; c[4] = ax[1]; c[5] = ax[2];
    }
  }
  __syncwarp();
}

__device__ __forceinline__ void cinert_mul(const float* ci, const float* v, float* f) {
  const float *w = v, *l = v + 3;
  f[0] = ci[0] * w[0] + ci[3] * w[1] + ci[4] * w[2] + (ci[7] * l[2] - ci[8] * l[1]);
  f[1] = ci[3] * w[0] + ci[1] * w[1] + ci[5] * w[2] + (ci[8] * l[0] - ci[6] * l[2]);
  f[2] = ci[4] * w[0] + ci[5] * w[1] + ci[2] * w[2] + (ci[6] * l[1] - ci[7] * l[0]);
  f[3] = ci[9] * l[0] - (ci[7] * w[2] - ci[8] * w[1]);
  f[4] = ci[9] * l[1] - (ci[8] * w[0] - ci[6] * w[2]);
  f[5] = ci[9] * l[2] - (ci[6] * w[1] - ci[7] * w[0]);
}

// composite rigid bodies and the joint-space mass matrix
__device__ __noinline__ void d_crb(Env& E) {
  const DevModelDesc& m = *E.md;
  const int* it = E.it;
  const float* ft = E.ft;
  float* ws = E.ws;
  float* crb = ws + m.w_crb;
  const float* cinert = ws + m.w_cinert;
  #pragma unroll 1
  for (int k = E.lane; k < 10 * m.nbody; k += 32) crb[k] = k < 10 ? 0.f : cinert[k];
  __syncwarp();
  for (int l = m.nlevel - 2; l >= 1; l--) {
    int s = ldi(it, m.i_level_start + l), e = ldi(it, m.i_level_start + l + 1);
    #pragma unroll 1
    for (int k = s + E.lane; k < e; k += 32) {
      int b = ldi(it, m.i_level_body + k);
      int c0 = ldi(it, m.i_child_start + b), c1 = ldi(it, m.i_child_start + b + 1);
      #pragma unroll 1
      for (int ci = c0; ci < c1; ci++) {
        int c = ldi(it, m.i_child_list + ci);
        for (int q = 0; q < 10; q++) crb[10 * b + q] += crb[10 * c + q];
      }
    }
    __syncwarp();
  }
  int nv = m.nv;
  float* M = ws + m.w_M;
  #pragma unroll 1
  for (int k = E.lane; k < nv * nv; k += 32) M[k] = 0;
  __syncwarp();
  const float* cdof = ws + m.w_cdof;
  #pragma unroll 1
  for (int i = E.lane; i < nv; i += 32) {
    float f[6];
    cinert_mul(crb + 10 * ldi(it, m.i_dof_bodyid + i), cdof + 6 * i, f);
    for (int j = i; j >= 0; j = ldi(it, m.i_dof_parentid + j)) {
      const float* cj = cdof + 6 * j;
      float s = f[0] * cj[0] + f[1] * cj[1] + f[2] * cj[2] + f[3] * cj[3] + f[4] * cj[4] + f[5] * cj[5];
      if (j == i) s += ldf(ft, m.f_dof_armature + i);
      M[i * nv + j] = s;
      M[j * nv + i] = s;
    }
  }
  __syncwarp();
}

__device__ __forceinline__ void cross_motion(const float* v, const float* u, float* r) {
  float a[3], b[3], c[3];
  cross3(v, u, c);
  cross3(v + 3, u, a);
  cross3(v, u + 3, b);
  r[0] = c[0]; r[1] = c[1]; r[2] = c[2];
  for (int k = 0; k < 3; k++) r[3 + k] = a[k] + b[k];
}
__device__ __forceinline__ void cross_force(const float* v, const float* f, float* r) {
  float a[3], b[3], c[3];
  cross3(v, f, a);
  cross3(v + 3, f + 3, b);
  cross3(v, f + 3, c);
  for (int k = 0; k < 3; k++) { r[k] = a[k] + b[k]; r[3 + k] = c[k]; }
}

// com velocities, cdof_dot, and the bias force (RNE with qacc = 0) into `bias`
__device__ __noinline__ void d_rne(Env& E, float* bias) {
  const DevModelDesc& m = *E.md;
  const int* it = E.it;
  float* ws = E.ws;
  const float* qv = ws + m.w_qvel;
  const float* cdof = ws + m.w_cdof;
  float* cvel = ws + m.w_cvel;
  float* cdd = ws + m.w_cdofdot;
  float* cacc = ws + m.w_cacc;
  float* cfrc = ws + m.w_crb;  // crb is dead after d_crb
  const float* cinert = ws + m.w_cinert;
  if (E.lane < 6) {
    cvel[E.lane] = 0;
    cacc[E.lane] = E.lane < 3 || (m.disableflags & (1 << 6)) ? 0.f : -m.gravity[E.lane - 3];
  }
  __syncwarp();
  #pragma unroll 1
  for (int l = 1; l < m.nlevel; l++) {
    int s = ldi(it, m.i_level_start + l), e = ldi(it, m.i_level_start + l + 1);
    #pragma unroll 1
    for (int k = s + E.lane; k < e; k += 32) {
      int b = ldi(it, m.i_level_body + k);
      int p = ldi(it, m.i_body_parentid + b);
      float cv[6], ca[6];
      for (int c = 0; c < 6; c++) { cv[c] = cvel[6 * p + c]; ca[c] = cacc[6 * p + c]; }
      int a = ldi(it, m.i_body_dofadr + b), n = ldi(it, m.i_body_dofnum + b);
      #pragma unroll 1
      for (int q = 0; q < n;) {
        int i = a + q;
        int t = ldi(it, m.i_jnt_type + ldi(it, m.i_dof_jntid + i));
        if (t == 0) {
          for (int s2 = 0; s2 < 3; s2++) {
            for (int c = 0; c < 6; c++) cdd[6 * (i + s2) + c] = 0;
            for (int c = 0; c < 6; c++) cv[c] += cdof[6 * (i + s2) + c] * qv[i + s2];
          }
          for (int s2 = 3; s2 < 6; s2++) cross_motion(cv, cdof + 6 * (i + s2), cdd + 6 * (i + s2));
          for (int s2 = 3; s2 < 6; s2++)
            for (int c = 0; c < 6; c++) cv[c] += cdof[6 * (i + s2) + c] * qv[i + s2];
          q += 6;
        } else if (t == 1) {
          for (int s2 = 0; s2 < 3; s2++) cross_motion(cv, cdof + 6 * (i + s2), cdd + 6 * (i + s2));
          for (int s2 = 0; s2 < 3; s2++)
            for (int c = 0; c < 6; c++) cv[c] += cdof[6 * (i + s2) + c] * qv[i + s2];
          q += 3;
        } else {
          cross_motion(cv, cdof + 6 * i, cdd + 6 * i);
          for (int c = 0; c < 6; c++) cv[c] += cdof[6 * i + c] * qv[i];
          q += 1;
        }
      }
      #pragma unroll 1
      for (int i = a; i < a + n; i++)
        for (int c = 0; c < 6; c++) ca[c] += cdd[6 * i + c] * qv[i];
      for (int c = 0; c < 6; c++) { cvel[6 * b + c] = cv[c]; cacc[6 * b + c] = ca[c]; }
    }
    __syncwarp();
  }
  #pragma unroll 1
  for (int b = E.lane; b < m.nbody; b += 32) {
    float Ia[6], Iv[6], vf[6];
    cinert_mul(cinert + 10 * b, cacc + 6 * b, Ia);
    cinert_mul(cinert + 10 * b, cvel + 6 * b, Iv);
    cross_force(cvel + 6 * b, Iv, vf);
    for (int c = 0; c < 6; c++) cfrc[6 * b + c] = Ia[c] + vf[c];
  }
  __syncwarp();
  for (int l = m.nlevel - 2; l >= 1; l--) {
    int s = ldi(it, m.i_level_start + l), e = ldi(it, m.i_level_start + l + 1);
    #pragma unroll 1
    for (int k = s + E.lane; k < e; k += 32) {
      int b = ldi(it, m.i_level_body + k);
      int c0 = ldi(it, m.i_child_start + b), c1 = ldi(it, m.i_child_start + b + 1);
      #pragma unroll 1
      for (int ci = c0; ci < c1; ci++) {
        int c = ldi(it, m.i_child_list + ci);
        for (int q = 0; q < 6; q++) cfrc[6 * b + q] += cfrc[6 * c + q];
      }
    }
    __syncwarp();
  }
  #pragma unroll 1
  for (int i = E.lane; i < m.nv; i += 32) {
    const float* f = cfrc + 6 * ldi(it, m.i_dof_bodyid + i);
    const float* c = cdof + 6 * i;
    bias[i] = c[0] * f[0] + c[1] * f[1] + c[2] * f[2] + c[3] * f[3] + c[4] * f[4] + c[5] * f[5];
  }
  __syncwarp();
}

// Tendons of this substep: length, velocity and Jacobian of every tendon
// into the persistent workspace (w_ten: per tendon [length, velocity,
// J(nv)]), computed once after the COM pass and read by the forces, the
// constraint rows and the sensors (reference: tendon.hpp emit_tendon_phase,
// MuJoCo mj_tendon).  Fixed tendons: length = sum coef * qpos, J = sum coef
// e_dof.  Spatial tendons: lane 0 walks the path (sites, wrapping sphere /
// cylinder geoms, pulley divisors) and lists its straight pieces; every
// lane then sums, for its dofs, piece direction x (Jacobian at the piece's
// end - Jacobian at its start), the tangent points of a wrap moving with the
// geom; velocity = J qvel.
__device__ __forceinline__ void d_site_world(const DevModelDesc& m, const int* it, const float* ft, const float* ws, int s, float* p) {
  const int b = ldi(it, m.i_site_body + s);
  const float q[4] = {ws[m.w_xquat + 4 * b], ws[m.w_xquat + 4 * b + 1], ws[m.w_xquat + 4 * b + 2], ws[m.w_xquat + 4 * b + 3]};
  const float l[3] = {ldf(ft, m.f_site + 3 * s), ldf(ft, m.f_site + 3 * s + 1), ldf(ft, m.f_site + 3 * s + 2)};
  float r[3];
  qrot(q, l, r);
  for (int k = 0; k < 3; k++) p[k] = ws[m.w_xpos + 3 * b + k] + r[k];
}

// lane 0: append the straight piece p0 (body b0) -> p1 (body b1), scaled
__device__ __forceinline__ void d_piece(float* seg, int& np, const float* p0, int b0, const float* p1, int b1, float scale) {
  float* q = seg + 9 * np++;
  for (int k = 0; k < 3; k++) { q[k] = p0[k]; q[3 + k] = p1[k]; }
  q[6] = __int_as_float(b0);
  q[7] = __int_as_float(b1);
  q[8] = scale;
}

__device__ __noinline__ void d_tendons(Env& E) {
  const DevModelDesc& m = *E.md;
  const int* it = E.it;
  const float* ft = E.ft;
  float* ws = E.ws;
  const int nv = m.nv, lane = E.lane;
  const float* qpos = ws + m.w_qpos;
  const float* qvel = ws + m.w_qvel;
  float* seg = ws + m.w_tseg;
  #pragma unroll 1
  for (int t = 0; t < m.ntendon; t++) {
    float* row = ws + m.w_ten + t * (nv + 2);
    const int adr = ldi(it, m.i_ten + 3 * t), num = ldi(it, m.i_ten + 3 * t + 1);
    int np = 0;
    float len = 0.f;
    if (lane == 0) {
      float scale = 1.f;
      #pragma unroll 1
      for (int w = adr; w < adr + num; w++) {
        const int* wi = it + m.i_wrap + 3 * w;
        const int ty = ldi(wi, 0);
        if (ty == 1) {
          len += ldf(ft, m.f_wrap + w) * qpos[ldi(wi, 2)];
        } else if (ty == 2) {
          scale = 1.f / ldf(ft, m.f_wrap + w);
        } else if (ty == 3 && w + 1 < adr + num) {
          const int* wn = wi + 3;
          const int tn = ldi(wn, 0);
          if (tn == 3) {
            float p0[3], p1[3];
            d_site_world(m, it, ft, ws, ldi(wi, 1), p0);
            d_site_world(m, it, ft, ws, ldi(wn, 1), p1);
            const float e[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
            len += scale * norm3(e);
            d_piece(seg, np, p0, ldi(wi, 2), p1, ldi(wn, 2), scale);
          } else if ((tn == 4 || tn == 5) && w + 2 < adr + num) {
            const int* w2 = wi + 6;
            const int g = ldi(wn, 1), ss = ldi(wn, 2), gb = ldi(it, m.i_geom_bodyid + g);
            float p0[3], p1[3], sp[3], t0[3], t1[3];
            d_site_world(m, it, ft, ws, ldi(wi, 1), p0);
            d_site_world(m, it, ft, ws, ldi(w2, 1), p1);
            if (ss >= 0) d_site_world(m, it, ft, ws, ss, sp);
            bool wrapped = false;
            const float full = mjbwrap::geom<float>(tn == 4 ? 2 : 5, ws + m.w_gxpos + 3 * g, ws + m.w_gxmat + 9 * g, ldf(ft, m.f_geom_size + 3 * g), p0,
                                                    p1, ss >= 0 ? sp : nullptr, t0, t1, wrapped);
            len += scale * full;
            if (!wrapped) {
              d_piece(seg, np, p0, ldi(wi, 2), p1, ldi(w2, 2), scale);
            } else {
              d_piece(seg, np, p0, ldi(wi, 2), t0, gb, scale);
              d_piece(seg, np, t1, gb, p1, ldi(w2, 2), scale);
            }
            w += 1;
          }
        }
      }
    }
    np = __shfl_sync(FULL_MASK, np, 0);
    len = __shfl_sync(FULL_MASK, len, 0);
    __syncwarp();
    float vpart = 0.f;
    #pragma unroll 1
    for (int i = lane; i < nv; i += 32) {
      float j = 0.f;
      #pragma unroll 1
      for (int w = adr; w < adr + num; w++)
        if (ldi(it, m.i_wrap + 3 * w) == 1 && ldi(it, m.i_wrap + 3 * w + 1) == i) j += ldf(ft, m.f_wrap + w);
      const int db = ldi(it, m.i_dof_bodyid + i), dsub = ldi(it, m.i_body_subtreesize + db);
      const float* cd = ws + m.w_cdof + 6 * i;
      #pragma unroll 1
      for (int p = 0; p < np; p++) {
        const float* q = seg + 9 * p;
        float e[3] = {q[3] - q[0], q[4] - q[1], q[5] - q[2]};
        const float l = norm3(e);
        if (l < 1e-12f) continue;
        for (int k = 0; k < 3; k++) e[k] /= l;
        for (int side = 0; side < 2; side++) {
          const int b = __float_as_int(q[6 + side]);
          if (b < db || b >= db + dsub) continue;
          const int root = ldi(it, m.i_body_rootid + b);
          const float* pt = q + 3 * side;
          const float off[3] = {pt[0] - ws[m.w_scom + 3 * root], pt[1] - ws[m.w_scom + 3 * root + 1], pt[2] - ws[m.w_scom + 3 * root + 2]};
          const float jp[3] = {cd[3] + cd[1] * off[2] - cd[2] * off[1], cd[4] + cd[2] * off[0] - cd[0] * off[2], cd[5] + cd[0] * off[1] - cd[1] * off[0]};
          j += (side ? 1.f : -1.f) * q[8] * (e[0] * jp[0] + e[1] * jp[1] + e[2] * jp[2]);
        }
      }
      row[2 + i] = j;
      vpart += j * qvel[i];
    }
    const float vel = warp_sum(vpart);
    if (lane == 0) {
      row[0] = len;
      row[1] = vel;
    }
    __syncwarp();
  }
}

__device__ __forceinline__ void d_tendon_lv(const DevModelDesc& m, const float* ws, int t, float& len, float& vel) {
  const float* row = ws + m.w_ten + t * (m.nv + 2);
  len = row[0];
  vel = row[1];
}

// Component of tendon t's Jacobian on dof i.
__device__ __forceinline__ float d_tendon_jac(const DevModelDesc& m, const float* ws, int t, int i) { return ws[m.w_ten + t * (m.nv + 2) + 2 + i]; }

// row[0..nv) = sg * (Jacobian of tendon t), written by one lane.
__device__ __forceinline__ void d_tendon_row(const DevModelDesc& m, const float* ws, int t, float sg, float* row) {
  const float* J = ws + m.w_ten + t * (m.nv + 2) + 2;
  #pragma unroll 1
  for (int c = 0; c < m.nv; c++) row[c] = sg * J[c];
}

// passive + actuation + smooth force
// Actuator forces, one lane per actuator: af[a] = gear * force of actuator
// a, at[a] = the dof it drives (joint transmission) or -(tendon + 1).  All
// actuators' table entries load at once; walking the actuators in sequence
// from every dof lane instead put one chain of cold table loads per actuator
// on the stage's critical path (18.7 K of the stage's 20.9 K cycles for the
// quadruped's 12 actuators).
__device__ __noinline__ void d_actuator_forces(Env& E, const StepParams& P, float* af, int* at) {
  const DevModelDesc& m = *E.md;
  const int* it = E.it;
  const float* ft = E.ft;
  const float* ws = E.ws;
  const float* qpos = ws + m.w_qpos;
  const float* qvel = ws + m.w_qvel;
  const float* ctrl = ws + m.w_ctrl;
  #pragma unroll 1
  for (int a = E.lane; a < m.nu; a += 32) {
    const int* ai = it + m.i_act + 7 * a;
    const float* fa = ft + m.f_act + 11 * a;
    const int dof = ldi(ai, 0), qa = ldi(ai, 1), gt = ldi(ai, 2), bt = ldi(ai, 3), cl = ldi(ai, 4), fl = ldi(ai, 5), ten = ldi(ai, 6);
    const float gear = ldf(fa, 0);
    float len, vel;
    if (ten >= 0) {
      d_tendon_lv(m, ws, ten, len, vel);
    } else {
      len = qpos[qa];
      vel = qvel[dof];
    }
    float c = ctrl[a];
    if (cl && !(m.disableflags & (1 << 7))) c = clampf(c, ldf(fa, 7), ldf(fa, 8));
    len *= gear;
    vel *= gear;
    const float gain = ldf(fa, 1) + (gt ? ldf(fa, 2) * len + ldf(fa, 3) * vel : 0.f);
    const float bs = bt ? ldf(fa, 4) + ldf(fa, 5) * len + ldf(fa, 6) * vel : 0.f;
    float force = gain * c + bs;
    if (P.rand_gain) force *= P.rand_gain[P.env_uadr[E.env] + a];
    if (fl) force = clampf(force, ldf(fa, 9), ldf(fa, 10));
    af[a] = gear * force;
    at[a] = ten >= 0 ? -(ten + 1) : dof;
  }
  __syncwarp();
}

__device__ __noinline__ void d_forces(Env& E, const StepParams& P, const float* bias) {
  const DevModelDesc& m = *E.md;
  const int* it = E.it;
  const float* ft = E.ft;
  float* ws = E.ws;
  const float* qpos = ws + m.w_qpos;
  const float* qvel = ws + m.w_qvel;
  const float* ctrl = ws + m.w_ctrl;
  float* qfs = ws + m.w_qfs;
  float* qfa = ws + m.w_qfa;
  // actuator forces lane-parallel into Newton's solver vectors 0-4 (free
  // during this stage) when nu forces and nu targets fit there
  float* af = ws + m.w_vec;
  int* at = reinterpret_cast<int*>(ws + m.w_vec) + m.nu;
  const bool lanepar = 2 * m.nu <= 5 * m.nv;
  if (lanepar && !(m.disableflags & (1 << 10))) d_actuator_forces(E, P, af, at);
  #pragma unroll 1
  for (int i = E.lane; i < m.nv; i += 32) {
    float pas = 0, act = 0;
    if (!(m.disableflags & (1 << 5))) {
      int j = ldi(it, m.i_dof_jntid + i);
      int t = ldi(it, m.i_jnt_type + j);
      float st = ldf(ft, m.f_jnt_stiffness + j);
      if ((t == 2 || t == 3) && st != 0.f) {
        int qa = ldi(it, m.i_jnt_qposadr + j);
        pas -= st * (qpos[qa] - ldf(ft, m.f_qpos_spring + qa));
      }
      pas -= ldf(ft, m.f_dof_damping + i) * qvel[i];
      // gravity compensation at each compensated body's COM, through cdof
      // (reference: forward.hpp:438-452)
      const int db = ldi(it, m.i_dof_bodyid + i), dsub = ldi(it, m.i_body_subtreesize + db);
      const int ngc = (m.disableflags & (1 << 6)) ? 0 : m.ngcomp;   // nothing to compensate without gravity
      #pragma unroll 1
      for (int k = 0; k < ngc; k++) {
        const int b = ldi(it, m.i_gcomp + k);
        if (b < db || b >= db + dsub) continue;
        const float mb = ldf(ft, m.f_body_mass + b) * ldf(ft, m.f_gcomp + k) * msc(P, E, b);
        const int root = ldi(it, m.i_body_rootid + b);
        const float* xi = ws + m.w_xipos + 3 * b;
        const float* rc = ws + m.w_scom + 3 * root;
        const float f[3] = {-mb * m.gravity[0], -mb * m.gravity[1], -mb * m.gravity[2]};
        const float o[3] = {xi[0] - rc[0], xi[1] - rc[1], xi[2] - rc[2]};
        float tq[3];
        cross3(o, f, tq);
        const float* cd = ws + m.w_cdof + 6 * i;
        pas += cd[0] * tq[0] + cd[1] * tq[1] + cd[2] * tq[2] + cd[3] * f[0] + cd[4] * f[1] + cd[5] * f[2];
      }
      // quadratic drag on the translational dofs of free joints (per env;
      // reference: forward.hpp:455-464)
      if (P.rand_drag) {
        #pragma unroll 1
        for (int k = 0; k < m.nfree; k++) {
          const int da = ldi(it, m.i_free + k);
          if (i < da || i >= da + 3) continue;
          const float vx = qvel[da], vy = qvel[da + 1], vz = qvel[da + 2];
          pas += -P.rand_drag[P.env_fadr[E.env] + k] * sqrtf(vx * vx + vy * vy + vz * vz) * qvel[i];
        }
      }
      // tendon spring with a dead band and damper, through J^T
      // (reference: tendon.hpp:360-377)
      #pragma unroll 1
      for (int k = 0; k < m.npten; k++) {
        const int t = ldi(it, m.i_pten + k);
        const float jt = d_tendon_jac(m, ws, t, i);
        if (jt == 0.f) continue;
        const float* tf = ft + m.f_ten + MJB_TEN_FLOATS * t;
        float len, vel;
        d_tendon_lv(m, ws, t, len, vel);
        const float kst = ldf(tf, TEN_STIFF), lo = ldf(tf, TEN_SPRLO), hi = ldf(tf, TEN_SPRHI);
        float f = 0.f;
        if (len > hi) f += kst * (hi - len);
        else if (len < lo) f += kst * (lo - len);
        f -= ldf(tf, TEN_DAMP) * vel;
        pas += jt * f;
      }
    }
    if (!(m.disableflags & (1 << 10))) {
      if (lanepar) {
        // sum of the posted actuator forces that drive dof i, in actuator order
        #pragma unroll 1
        for (int a = 0; a < m.nu; a++) {
          const int t = at[a];
          if (t >= 0) {
            if (t == i) act += af[a];
          } else {
            const float moment = d_tendon_jac(m, ws, -t - 1, i);
            if (moment != 0.f) act += moment * af[a];
          }
        }
      } else {
        #pragma unroll 1
        for (int a = 0; a < m.nu; a++) {
          const int* ai = it + m.i_act + 7 * a;
          const int ten = ldi(ai, 6);
          float moment = 1.f, len, vel;
          if (ten >= 0) {
            // tendon transmission: length / velocity / moment from the tendon
            moment = d_tendon_jac(m, ws, ten, i);
            if (moment == 0.f) continue;
            d_tendon_lv(m, ws, ten, len, vel);
          } else {
            if (ldi(ai, 0) != i) continue;
            len = qpos[ldi(ai, 1)];
            vel = qvel[i];
          }
          const float* fa = ft + m.f_act + 11 * a;
          float gear = ldf(fa, 0);
          float c = ctrl[a];
          if (ldi(ai, 4) && !(m.disableflags & (1 << 7))) c = clampf(c, ldf(fa, 7), ldf(fa, 8));
          len *= gear;
          vel *= gear;
          float gain = ldf(fa, 1) + (ldi(ai, 2) ? ldf(fa, 2) * len + ldf(fa, 3) * vel : 0.f);
          float bs = ldi(ai, 3) ? ldf(fa, 4) + ldf(fa, 5) * len + ldf(fa, 6) * vel : 0.f;
          float force = gain * c + bs;
          if (P.rand_gain) force *= P.rand_gain[P.env_uadr[E.env] + a];
          if (ldi(ai, 5)) force = clampf(force, ldf(fa, 9), ldf(fa, 10));
          act += gear * moment * force;
        }
      }
    }
    qfa[i] = act;
    qfs[i] = pas - bias[i] + act;
  }
  __syncwarp();
}

}  // namespace mjbdev
