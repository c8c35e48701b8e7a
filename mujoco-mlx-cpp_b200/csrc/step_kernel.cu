// Fused physics-step kernel for sm_100a: one warp per environment, nsub
// substeps per launch, every intermediate in the warp's shared-memory
// workspace.  HBM traffic per env-substep is the state record only (qpos,
// qvel, ctrl, warm-start qacc in; qpos, qvel, qacc out) -- the reference runs
// six separate dispatches per substep that round-trip kinematics, mass
// matrix, contacts and solver scratch through device memory
// (src/batched.cpp:980-1228).
#include <cuda_runtime.h>

#include <mutex>

#include "dev_nn.cuh"
#include "dev_solver.cuh"
#include "step_params.h"

using namespace mjbdev;

namespace {

__device__ __forceinline__ bool badval(float v) { return !(fabsf(v) <= 1e10f); }

__device__ __noinline__ void reset_env(Env& E) {
  const DevModelDesc& m = *E.md;
  float* ws = E.ws;
  #pragma unroll 1
  for (int i = E.lane; i < m.nq; i += 32) ws[m.w_qpos + i] = ldf(E.ft, m.f_qpos0 + i);
  #pragma unroll 1
  for (int i = E.lane; i < m.nv; i += 32) {
    ws[m.w_qvel + i] = 0;
    ws[m.w_xwarm + i] = 0;
    ws[m.w_x + i] = 0;
  }
  __syncwarp();
}

// contact wrench per body in com-based coordinates (torque about the
// subtree COM of the body's root, force), accumulated by lane 0
__device__ __noinline__ void record_cfrc(Env& E, const StepParams& P, int ncon, int nefc, float* out) {
  const DevModelDesc& m = *E.md;
  const float* efc = E.ws + m.w_efc;
  const int ne = m.nefc_max;
  const float* con = E.ws + m.w_con;
  const float* scom = E.ws + m.w_scom;
  #pragma unroll 1
  for (int k = E.lane; k < 6 * m.nbody; k += 32) out[k] = 0;
  __syncwarp();
  if (E.lane == 0) {
    int r = 0;
    while (r < nefc) {
      int c = (int)efc[EFC_CON * ne + r];
      if (c < 0) { r++; continue; }
      const float* cr = con + MJB_CONTACT_FLOATS * c;
      int dim = (int)cr[14];
      const bool ell = (int)efc[EFC_TYPE * ne + r] == ROW_ELLIPTIC;
      int nr = dim == 1 ? 1 : ell ? dim : 2 * (dim - 1);
      int p = (int)cr[13];
      const float* pf = E.ft + m.f_pair + 16 * p;
      float fs = P.rand_friction ? P.rand_friction[E.env] : 1.f;
      float fn = 0, ft[5] = {0, 0, 0, 0, 0};
      if (ell) {
        // elliptic: the normal row's force and one force per friction direction
        fn = efc[EFC_FORCE * ne + r];
        for (int d = 0; d + 1 < dim; d++) ft[d] = efc[EFC_FORCE * ne + r + 1 + d];
      } else {
        #pragma unroll 1
        for (int q = 0; q < nr; q++) fn += efc[EFC_FORCE * ne + r + q];
        for (int d = 0; d + 1 < dim; d++)
          ft[d] = ldf(pf, 2 + d) * fs * (efc[EFC_FORCE * ne + r + 2 * d] - efc[EFC_FORCE * ne + r + 2 * d + 1]);
      }
      const float* n = cr + 3;
      const float* t1 = cr + 6;
      const float* t2 = cr + 9;
      float F[3], T[3];
      for (int k = 0; k < 3; k++) {
        F[k] = fn * n[k] + ft[0] * t1[k] + ft[1] * t2[k];
        T[k] = ft[2] * n[k] + ft[3] * t1[k] + ft[4] * t2[k];
      }
      int b1 = ldi(E.it, m.i_pair + 6 * p + 2), b2 = ldi(E.it, m.i_pair + 6 * p + 3);
      for (int side = 0; side < 2; side++) {
        int b = side == 0 ? b2 : b1;
        float sg = side == 0 ? 1.f : -1.f;
        int root = ldi(E.it, m.i_body_rootid + b);
        float off[3] = {cr[0] - scom[3 * root], cr[1] - scom[3 * root + 1], cr[2] - scom[3 * root + 2]}, tq[3];
        cross3(off, F, tq);
        for (int k = 0; k < 3; k++) {
          out[6 * b + k] += sg * (tq[k] + T[k]);
          out[6 * b + 3 + k] += sg * F[k];
        }
      }
      r += nr;
    }
  }
  __syncwarp();
}

}  // namespace

extern __shared__ float mjb_smem[];

namespace {

__device__ __noinline__ void record_debug(Env& E, const StepParams& P, int ncon, int nefc, const float* qfc) {
  const DevModelDesc& m = *E.md;
  const float* ws = E.ws;
  const int lane = E.lane, nv = m.nv, env = E.env;
  float* dc = P.dbg_contacts + (size_t)env * P.dbg_ncon_max * MJB_CONTACT_FLOATS;
  int nc = ncon < P.dbg_ncon_max ? ncon : P.dbg_ncon_max;
#pragma unroll 1
  for (int k = lane; k < nc * MJB_CONTACT_FLOATS; k += 32) dc[k] = ws[m.w_con + k];
  float* de = P.dbg_efc + (size_t)env * P.dbg_nefc_max * 4;
  int ne = nefc < P.dbg_nefc_max ? nefc : P.dbg_nefc_max;
#pragma unroll 1
  for (int r = lane; r < ne; r += 32) {
    EfcRef e{const_cast<float*>(ws) + m.w_efc + r, m.nefc_max};
    de[4 * r] = e[EFC_TYPE];
    de[4 * r + 1] = e[EFC_FORCE];
    de[4 * r + 2] = e[EFC_D];
    de[4 * r + 3] = e[EFC_AREF];
  }
  float* dv = P.dbg_vec + (size_t)env * 4 * P.dbg_nv_max;
#pragma unroll 1
  for (int k = lane; k < nv; k += 32) {
    dv[k] = ws[m.w_qas + k];
    dv[P.dbg_nv_max + k] = ws[m.w_qfs + k];
    dv[2 * P.dbg_nv_max + k] = ws[m.w_x + k];
    dv[3 * P.dbg_nv_max + k] = qfc[k];
  }
  __syncwarp();
}

__device__ __noinline__ void record_kin(Env& E, const StepParams& P, int badr) {
  const DevModelDesc& m = *E.md;
  const float* ws = E.ws;
  const int lane = E.lane;
#pragma unroll 1
  for (int k = lane; k < 3 * m.nbody; k += 32) {
    P.rec_xpos[3 * badr + k] = ws[m.w_xpos + k];
    P.rec_scom[3 * badr + k] = ws[m.w_scom + k];
  }
#pragma unroll 1
  for (int k = lane; k < 4 * m.nbody; k += 32) P.rec_xquat[4 * badr + k] = ws[m.w_xquat + k];
#pragma unroll 1
  for (int k = lane; k < 10 * m.nbody; k += 32) P.rec_cinert[10 * badr + k] = ws[m.w_cinert + k];
}

__device__ __noinline__ void record_dyn(Env& E, const StepParams& P, int badr, int vadr) {
  const DevModelDesc& m = *E.md;
  const float* ws = E.ws;
  const int lane = E.lane;
#pragma unroll 1
  for (int k = lane; k < 6 * m.nbody; k += 32) P.rec_cvel[6 * badr + k] = ws[m.w_cvel + k];
#pragma unroll 1
  for (int k = lane; k < m.nv; k += 32) P.rec_qfrc_actuator[vadr + k] = ws[m.w_qfa + k];
}

// Sensors at the substep's start state (reference: sensor_compute,
// sensor.cpp:265-356; MuJoCo's position / velocity stage formulas), one lane
// per sensor, after RNE while kinematics, cvel and qfrc_actuator are in the
// workspace.  write: store sensordata (last substep); save: store each
// accelerometer frame's world linear velocity as the next one's previous
// value.  prev_ok: the stored previous velocity is valid.
__device__ __noinline__ void record_sensors(Env& E, const StepParams& P, bool write, bool save, bool prev_ok) {
  const DevModelDesc& m = *E.md;
  const int* it = E.it;
  const float* ft = E.ft;
  const float* ws = E.ws;
  const float* qpos = ws + m.w_qpos;
  const float* qvel = ws + m.w_qvel;
  float* out = write ? P.sensordata + P.env_sadr[E.env] : nullptr;
  float* prev = P.sens_prev ? P.sens_prev + P.env_aadr[E.env] : nullptr;
#pragma unroll 1
  for (int s = E.lane; s < m.nsensor; s += 32) {
    const int* si = it + m.i_sensor + MJB_SENSOR_INTS * s;
    const float* sf = ft + m.f_sensor + MJB_SENSOR_FLOATS * s;
    const int type = ldi(si, 0), adr = ldi(si, 1), dim = ldi(si, 2), a = ldi(si, 5), b = ldi(si, 6), slot = ldi(si, 7);
    if (!write && type != 1) continue;   // history only: accelerometers
    float y[4] = {0.f, 0.f, 0.f, 0.f};
    switch (type) {
      case 9: y[0] = qpos[a]; break;                      // jointpos
      case 10: y[0] = qvel[a]; break;                     // jointvel
      case 16: y[0] = ws[m.w_qfa + a]; break;             // jointactuatorfrc
      case 11: case 12: {                                 // tendonpos / tendonvel
        float len, vel;
        d_tendon_lv(m, ws, a, len, vel);
        y[0] = type == 11 ? len : vel;
        break;
      }
      case 13: case 14: {                                 // actuatorpos / actuatorvel
        float len, vel;
        if (b < 0) d_tendon_lv(m, ws, a, len, vel);
        else { len = qpos[a]; vel = qvel[b]; }
        y[0] = ldf(sf, 7) * (type == 13 ? len : vel);
        break;
      }
      case 18: {                                          // ballquat
        float q[4] = {qpos[a], qpos[a + 1], qpos[a + 2], qpos[a + 3]};
        const float inv = rsqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        for (int k = 0; k < 4; k++) y[k] = q[k] * inv;
        break;
      }
      case 19: for (int k = 0; k < 3; k++) y[k] = qvel[a + k]; break;                  // ballangvel
      case 35: for (int k = 0; k < 3; k++) y[k] = ws[m.w_scom + 3 * a + k]; break;     // subtreecom
      case 1: case 2: case 3: case 6: case 26: case 27: case 28: case 29: case 30: case 31: case 32: {
        // object frame: body pose composed with the object's local frame
        const int body = ldi(si, 3), root = ldi(si, 4);
        const float* bp = ws + m.w_xpos + 3 * body;
        const float bq[4] = {ws[m.w_xquat + 4 * body], ws[m.w_xquat + 4 * body + 1], ws[m.w_xquat + 4 * body + 2], ws[m.w_xquat + 4 * body + 3]};
        const float lp[3] = {ldf(sf, 0), ldf(sf, 1), ldf(sf, 2)}, lq[4] = {ldf(sf, 3), ldf(sf, 4), ldf(sf, 5), ldf(sf, 6)};
        float off[3], pos[3], quat[4], R[9];
        qrot(bq, lp, off);
        for (int k = 0; k < 3; k++) pos[k] = bp[k] + off[k];
        qmul(bq, lq, quat);
        q2mat(quat, R);
        // velocity of the frame origin: cvel moved from the root subtree COM
        const float* cv = ws + m.w_cvel + 6 * body;
        const float w[3] = {cv[0], cv[1], cv[2]};
        const float r[3] = {pos[0] - ws[m.w_scom + 3 * root], pos[1] - ws[m.w_scom + 3 * root + 1], pos[2] - ws[m.w_scom + 3 * root + 2]};
        float wxr[3], v[3];
        cross3(w, r, wxr);
        for (int k = 0; k < 3; k++) v[k] = cv[3 + k] + wxr[k];
        switch (type) {
          case 26: for (int k = 0; k < 3; k++) y[k] = pos[k]; break;
          case 27: { const float sg = quat[0] < 0.f ? -1.f : 1.f; for (int k = 0; k < 4; k++) y[k] = sg * quat[k]; break; }
          case 28: case 29: case 30: for (int k = 0; k < 3; k++) y[k] = R[3 * k + (type - 28)]; break;
          case 31: for (int k = 0; k < 3; k++) y[k] = v[k]; break;
          case 32: for (int k = 0; k < 3; k++) y[k] = w[k]; break;
          case 3: mulmatT(R, w, y); break;
          case 2: mulmatT(R, v, y); break;
          case 6: mulmatT(R, m.magnetic, y); break;
          case 1: {
            // one-substep difference of the world linear velocity, minus gravity, in the site frame
            float acc[3] = {0.f, 0.f, 0.f};
            if (prev_ok)
              for (int k = 0; k < 3; k++) acc[k] = (v[k] - prev[3 * slot + k]) / m.timestep;
            for (int k = 0; k < 3; k++) acc[k] -= m.gravity[k];
            mulmatT(R, acc, y);
            if (save)
              for (int k = 0; k < 3; k++) prev[3 * slot + k] = v[k];
            break;
          }
          default: break;
        }
        break;
      }
      default: break;   // outside the batched set: zeros
    }
    if (write)
      for (int k = 0; k < dim; k++) out[adr + k] = y[k];
  }
  __syncwarp();
}

// unconstrained acceleration qacc_smooth = M^-1 qfrc_smooth
__device__ __noinline__ void d_qacc_smooth(Env& E) {
  const DevModelDesc& m = *E.md;
  float* ws = E.ws;
  const int nv = m.nv, lane = E.lane;
  float* H = ws + m.w_H;
#pragma unroll 1
  for (int k = lane; k < nv; k += 32) ws[m.w_qas + k] = ws[m.w_qfs + k];
  __syncwarp();
  float* idiag = ws + m.w_vec + 8 * nv;
  if (nv <= 32) {
    // explicit inverse: H <- M^-1 (the Newton solver starts from it),
    // qacc_smooth = M^-1 qfrc_smooth
    d_factor(E, nullptr, 0, nullptr, 0.f, H, idiag, false, nullptr, 0, true);
    const float a = d_inv_apply(H, nv, m.ldh, H + nv * m.ldh, ws + m.w_qfs, lane);
    if (lane < nv) ws[m.w_qas + lane] = a;
    __syncwarp();
    return;
  }
  d_factor(E, nullptr, 0, nullptr, 0.f, H, idiag);
  d_chol_solve(H, idiag, nv, m.ldh, ws + m.w_qas, lane);
}

// bad-acceleration check, implicit-damping solve, warm-start save, integration.
// Returns false if the env was reset.
__device__ __noinline__ bool d_finish(Env& E, const float* qfc, float* acc) {
  const DevModelDesc& m = *E.md;
  float* ws = E.ws;
  const int nv = m.nv, lane = E.lane;
  const float* x = ws + m.w_x;
  bool badacc = false;
#pragma unroll 1
  for (int i = lane; i < nv; i += 32) badacc |= badval(x[i]);
  if (__any_sync(FULL_MASK, badacc)) {
    env_status(E, MJB_STATUS_BADQACC);
    reset_env(E);
    return false;
  }
  const float* a = x;
  if (m.implicit) {
    float* H = ws + m.w_H;
#pragma unroll 1
    for (int k = lane; k < nv; k += 32) acc[k] = ws[m.w_qfs + k] + qfc[k];
    __syncwarp();
    float* idiag = ws + m.w_vec + 8 * nv;
    d_factor(E, nullptr, 0, E.ft + m.f_dof_damping_implicit, m.timestep, H, idiag);
    d_chol_solve(H, idiag, nv, m.ldh, acc, lane);
    a = acc;
  }
#pragma unroll 1
  for (int k = lane; k < nv; k += 32) ws[m.w_xwarm + k] = x[k];
  __syncwarp();
  d_integrate(E, a);
  return true;
}

// Feature row of the learned warm start, written after a substep: the state
// the next substep starts from (qpos without the skipped leading
// coordinates, qvel), the converged acceleration of this substep, and the
// normal and distance of the first MJB_FEAT_CONTACTS contacts.
// Per-body rows (P.feat_body): lane per body, contacts scanned in order.
__device__ __noinline__ void write_body_features(Env& E, const StepParams& P, int ncon) {
  const DevModelDesc& m = *E.md;
  const float* ws = E.ws;
  const int nb = m.nbody - 1;
  float* base = P.features + (size_t)E.env * nb * P.feat_stride;
#pragma unroll 1
  for (int b = E.lane; b < nb; b += 32) {
    const int body = b + 1, j = ldi(E.it, m.i_body_jntadr + body);
    const int qa = ldi(E.it, m.i_jnt_qposadr + j), va = ldi(E.it, m.i_jnt_dofadr + j);
    float* f = base + (size_t)b * P.feat_stride;
    const float* q = ws + m.w_qpos + qa;
    f[0] = q[2];
    for (int k = 0; k < 4; k++) f[1 + k] = q[3 + k];
    for (int k = 0; k < 6; k++) {
      f[5 + k] = ws[m.w_qvel + va + k];
      f[11 + k] = ws[m.w_x + va + k];
    }
    int n = 0;
#pragma unroll 1
    for (int c = 0; c < ncon && n < MJB_FEAT_BODY_CONTACTS; c++) {
      const float* cr = ws + m.w_con + c * MJB_CONTACT_FLOATS;
      const int p = (int)cr[13];
      const int b1 = ldi(E.it, m.i_pair + 6 * p + 2), b2 = ldi(E.it, m.i_pair + 6 * p + 3);
      if (b1 != body && b2 != body) continue;
      const float sg = b2 == body ? 1.f : -1.f;   // the normal points from geom 1 to geom 2
      float* o = f + 17 + 7 * n;
      for (int k = 0; k < 3; k++) {
        o[k] = sg * cr[3 + k];
        o[4 + k] = cr[k] - q[k];
      }
      o[3] = cr[12];
      n++;
    }
    for (int k = 17 + 7 * n; k < MJB_FEAT_BODY; k++) f[k] = 0.f;
  }
}

__device__ __noinline__ void write_features(Env& E, const StepParams& P, int ncon) {
  if (P.feat_body) {
    write_body_features(E, P, ncon);
    return;
  }
  const DevModelDesc& m = *E.md;
  const float* ws = E.ws;
  const int nv = m.nv, lane = E.lane;
  float* f = P.features + (size_t)E.env * P.feat_stride;
  const int nqf = m.nq - P.feat_qskip;
#pragma unroll 1
  for (int i = lane; i < nqf; i += 32) f[i] = ws[m.w_qpos + P.feat_qskip + i];
  f += nqf;
#pragma unroll 1
  for (int i = lane; i < nv; i += 32) {
    f[i] = ws[m.w_qvel + i];
    f[nv + i] = ws[m.w_x + i];
  }
  f += 2 * nv;
#pragma unroll 1
  for (int k = lane; k < 4 * MJB_FEAT_CONTACTS; k += 32) {
    const int c = k >> 2, q = k & 3;
    float v = 0.f;
    if (c < ncon) {
      const float* con = ws + m.w_con + c * MJB_CONTACT_FLOATS;
      v = q < 3 ? con[3 + q] : con[12];
    }
    f[k] = v;
  }
}

__device__ __noinline__ bool check_state(Env& E) {
  const DevModelDesc& m = *E.md;
  const float* ws = E.ws;
  bool bad = false;
#pragma unroll 1
  for (int i = E.lane; i < m.nq; i += 32) bad |= badval(ws[m.w_qpos + i]);
#pragma unroll 1
  for (int i = E.lane; i < m.nv; i += 32) bad |= badval(ws[m.w_qvel + i]);
  if (__any_sync(FULL_MASK, bad)) {
    env_status(E, MJB_STATUS_BADSTATE);
    reset_env(E);
    return true;
  }
  return false;
}

}  // namespace

namespace {

// Feature row of the env (training pairs and / or the MLP's input row), then
// with fused = true the MLP over the CTA's envs.  Every warp of a lockstep
// CTA calls it with fused = true (block barriers inside); rows use warp 0's
// descriptor, which always belongs to a valid env.
__device__ __noinline__ void d_nn_stage(const Env& E, const StepParams& P, int ncon, bool valid, int s, bool last, bool fused) {
  float* raw = (P.pair_x && valid) ? P.pair_x + ((size_t)s * P.num_envs + E.env) * P.nn_in_raw
                                   : (last && P.nn_feat_out && valid) ? P.nn_feat_out + (size_t)E.env * P.nn_in_raw : nullptr;
  if (!fused) {
    d_nn_features(E, P, ncon, true, raw);
    return;
  }
  const int W = blockDim.x >> 5, warp = threadIdx.x >> 5;
  Env En = E;
  En.md = reinterpret_cast<const DevModelDesc*>(mjb_smem);
  d_nn_features(En, P, ncon, valid, raw);
  d_nn_infer(P, *En.md, mjb_smem + W * P.desc_words, W, warp, E.lane);
}

}  // namespace

// SM cycle counter read that the compiler keeps in place relative to the
// memory operations around it.
__device__ __forceinline__ long long stage_clock() {
  long long t;
  asm volatile("mov.u64 %0, %%clock64;" : "=l"(t) : : "memory");
  return t;
}

// Two execution modes share the stage functions:
//  * independent warps (P.lockstep == 0): each warp takes envs from the
//    persistent queue and runs all stages on its own;
//  * block lockstep (P.lockstep == 1): the warps of a CTA process a group of
//    envs together and meet at a barrier after every stage, so all warps of
//    the CTA execute the same stage code at the same time (instruction-cache
//    locality); envs whose Newton solve ends early wait at the barrier.
template <bool CVX>
__global__ void __launch_bounds__(512) mjb_step_kernel(const __grid_constant__ StepParams P) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int W = blockDim.x >> 5;
  const bool lockstep = P.lockstep != 0;
  // the fused warm start is compiled into the instance without the GJK / EPA
  // collider and elliptic solver only (the host refuses it for those models)
  const bool nnfused = !CVX && lockstep && P.nn_w[0] != nullptr && P.gws == nullptr;
  int* dsm = reinterpret_cast<int*>(mjb_smem) + warp * P.desc_words;
  float* ws = P.gws ? P.gws + ((size_t)blockIdx.x * W + warp) * P.ws_stride : mjb_smem + W * P.desc_words + warp * P.ws_stride;
  // optional per-stage timing: thread 0 of each CTA accumulates the clock
  // between consecutive stage barriers
  // Stage clocks: each warp's lane 0 posts its arrival time at a stage
  // barrier into tarr[tpar] (atomicMax), so after the barrier the slot holds
  // the moment the last warp arrived, i.e. when the barrier completed.  (A
  // clock read placed after the barrier can be issued before the barrier
  // completes, which moves barrier waits into the next stage's bucket.)
  // The two slots alternate; each is cleared by thread 0 right after it is
  // read, one barrier before its next use.
  __shared__ unsigned long long tarr[2];
  const bool stimed = lockstep && P.stage_cycles != nullptr;
  const bool timing = stimed && threadIdx.x == 0;
  unsigned long long tstage[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  long long tlast = timing ? stage_clock() : 0;
  int stage_id = 0, tpar = 0;
  if (stimed) {
    if (threadIdx.x == 0) tarr[0] = tarr[1] = 0ull;
    __syncthreads();
  }
#define TIMED_BARRIER(bucket)                                                        \
  do {                                                                               \
    __syncwarp();                                                                    \
    if (stimed && lane == 0) atomicMax(&tarr[tpar], (unsigned long long)stage_clock()); \
    __syncthreads();                                                                 \
    if (timing) {                                                                    \
      const long long t_ = (long long)tarr[tpar];                                    \
      tstage[(bucket) & 7] += (unsigned long long)(t_ - tlast);                      \
      tlast = t_;                                                                    \
      tarr[tpar] = 0ull;                                                             \
    }                                                                                \
    tpar ^= 1;                                                                       \
  } while (0)
#define STAGE_SYNC()                 \
  do {                               \
    if (lockstep) TIMED_BARRIER(stage_id); \
    stage_id++;                      \
  } while (0)

  // the model int table, copied into shared memory after the workspaces when
  // the host left room for it (P.itab_smem words)
  const int* itab = P.itab;
  if (P.itab_smem) {
    int* its = reinterpret_cast<int*>(mjb_smem + W * P.desc_words + (P.gws ? 0 : W * P.ws_stride));
#pragma unroll 1
    for (int k = threadIdx.x; k < P.itab_smem; k += blockDim.x) its[k] = __ldg(P.itab + k);
    __syncthreads();
    itab = its;
  }
  int group = blockIdx.x;
  int env = blockIdx.x * W + warp;
  if (!lockstep && P.work_counter) {
    int e = 0;
    if (lane == 0) e = atomicAdd(P.work_counter, 1);
    env = __shfl_sync(FULL_MASK, e, 0);
  }
  for (;;) {
    if (lockstep) {
      if (group * W >= P.num_envs) break;
      env = group * W + warp;
    } else if (env >= P.num_envs) {
      break;
    }
    const bool valid = env < P.num_envs;
    // the warp's context lives in its shared-memory slot after the
    // descriptor copy; lane 0 fills it for this env
    Env& E = *reinterpret_cast<Env*>(dsm + MJB_DESC_COPY_WORDS);
    __syncwarp();
    if (lane == 0) {
      E.it = itab;
      E.ft = P.ftab;
      E.ws = ws;
      E.env = env;
      E.status = 0;
      E.md = reinterpret_cast<const DevModelDesc*>(dsm);
    }
    __syncwarp();
    int qadr = 0, vadr = 0, badr = 0, nv = 0;
    if (P.poison_workspace) {
      // test aid: any read of the workspace before it is written in this
      // launch shows up as NaN (the state check then resets the env)
#pragma unroll 1
      for (int k = lane; k < P.ws_stride; k += 32) ws[k] = __int_as_float(0x7fc00000);
      __syncwarp();
    }
    if (valid) {
      const int* src = reinterpret_cast<const int*>(P.models + P.env_model[env]);
#pragma unroll 1
      for (int k = lane; k < MJB_DESC_COPY_WORDS; k += 32) dsm[k] = __ldg(src + k);
      __syncwarp();
      const DevModelDesc& m = *E.md;
      nv = m.nv;
      qadr = P.env_qadr[env];
      vadr = P.env_vadr[env];
      badr = P.env_badr[env];
      const int uadr = P.env_uadr[env];
#pragma unroll 1
      for (int i = lane; i < m.nq; i += 32) ws[m.w_qpos + i] = P.qpos[qadr + i];
#pragma unroll 1
      for (int i = lane; i < nv; i += 32) {
        ws[m.w_qvel + i] = P.qvel[vadr + i];
        ws[m.w_xwarm + i] = P.qacc_warm[vadr + i];
      }
#pragma unroll 1
      for (int i = lane; i < m.nu; i += 32) ws[m.w_ctrl + i] = P.ctrl[uadr + i];
      __syncwarp();
    }
    const int max_iter = valid ? (P.max_iter > 0 ? P.max_iter : E.md->iterations) : 0;
    // accelerometer history of this env is valid (cleared by resets)
    bool sens_ok = valid && P.sens_valid ? P.sens_valid[env] != 0 : false;
    const bool sensors = valid && E.md->nsensor > 0 && P.env_sadr;
    int nsum = 0, nmax = 0, ncon = 0, nefc = 0, choice = 0;
    float* vec = valid ? ws + E.md->w_vec : ws;
    float* qfc = vec + 5 * nv;
    float* acc = vec + 6 * nv;
    float* bias = vec + 7 * nv;
#pragma unroll 1
    for (int s = 0; s < P.nsub; s++) {
      const bool last = s == P.nsub - 1;
      stage_id = 0;
      if (valid) {
        if (check_state(E)) sens_ok = false;
        d_kinematics(E);
      }
      STAGE_SYNC();
      if (valid) ncon = d_collide<CVX>(E);
      STAGE_SYNC();
      if (valid) {
        d_com(E, P);
        if (last && P.rec_xpos) record_kin(E, P, badr);
        d_crb(E);
      }
      STAGE_SYNC();
      if (valid) {
        d_rne(E, bias);
        if (E.md->ntendon) d_tendons(E);
        d_forces(E, P, bias);
        if (last && P.rec_xpos) record_dyn(E, P, badr, vadr);
        if (sensors) {
          const bool write = last && P.sensordata, save = P.sens_prev && s >= P.nsub - 2;
          if (write || save) record_sensors(E, P, write, save, sens_ok);
          if (save) sens_ok = true;
        }
      }
      STAGE_SYNC();
      if (valid) d_qacc_smooth(E);
      STAGE_SYNC();
      if (valid) nefc = d_constraints<CVX>(E, P, ncon);
      STAGE_SYNC();
      // fused learned warm start: feature rows of this substep, then the MLP
      // over the CTA's envs (block barriers inside: every warp takes part)
      if constexpr (!CVX) {
        if (nnfused || (P.pair_x && valid)) {
          d_nn_stage(E, P, ncon, valid, s, last, nnfused);
          // stage clock bucket 6: the fused inference (one more barrier, only while timing)
          if (nnfused && stimed) TIMED_BARRIER(6);
        }
      }
      if (valid) {
        // a caller / separately inferred prediction serves the launch's first substep; the fused one every substep
        const float* xpred = nnfused ? ws + E.md->w_vec + 7 * nv : (P.qacc_pred && s == 0) ? P.qacc_pred + vadr : nullptr;
        // inverse mode for small models without elliptic cones; H still
        // holds the unconstrained solve's M^-1 (nv <= 32) unless the learned
        // warm start's features took its slot
        const bool inv = !(CVX && E.md->cone == 1) && nv <= 32 && nefc <= 128;
        const bool hm = P.nn_w[0] == nullptr;
        int it = inv ? d_newton<CVX, true>(E, P, nefc, max_iter, xpred, choice, hm) : d_newton<CVX, false>(E, P, nefc, max_iter, xpred, choice, hm);
        nsum += it;
        nmax = it > nmax ? it : nmax;
        if (P.pair_t) {
          float* tr = P.pair_t + ((size_t)s * P.num_envs + env) * nv;
#pragma unroll 1
          for (int k = lane; k < nv; k += 32) tr[k] = ws[E.md->w_x + k] - ws[E.md->w_xwarm + k];
        }
        if (last && nnfused && P.nn_pred_out) {
#pragma unroll 1
          for (int k = lane; k < nv; k += 32) P.nn_pred_out[vadr + k] = ws[E.md->w_vec + 7 * nv + k];
        }
      }
      // Barrier after Newton: the CTA's slowest solves finish while the other
      // warps wait, so only Newton code competes for the instruction cache
      // (letting early warps run on through integration and the next
      // kinematics instead measured 4.83 against 4.30 ms per 16,384-env
      // launch).  Stage clock bucket 7.
      if (lockstep) TIMED_BARRIER(7);
      if (valid) {
        d_jtf(E, nefc, qfc);
        if (last && P.dbg_contacts) record_debug(E, P, ncon, nefc, qfc);
        if (last && P.rec_cfrc_ext) record_cfrc(E, P, ncon, nefc, P.rec_cfrc_ext + 6 * badr);
        if (last && P.rec_qacc) {
#pragma unroll 1
          for (int k = lane; k < nv; k += 32) P.rec_qacc[vadr + k] = ws[E.md->w_x + k];
        }
        d_finish(E, qfc, acc);
        if (P.features) write_features(E, P, ncon);
      }
    }
    if (valid) {
      const DevModelDesc& m = *E.md;
#pragma unroll 1
      for (int i = lane; i < m.nq; i += 32) P.qpos[qadr + i] = ws[m.w_qpos + i];
#pragma unroll 1
      for (int i = lane; i < nv; i += 32) {
        P.qvel[vadr + i] = ws[m.w_qvel + i];
        P.qacc_warm[vadr + i] = ws[m.w_xwarm + i];
      }
      if (lane == 0) {
        if (P.status) P.status[env] = E.status;
        if (P.niter_sum) P.niter_sum[env] = P.stats_accumulate ? P.niter_sum[env] + nsum : nsum;
        if (P.niter_max) P.niter_max[env] = P.stats_accumulate ? max(P.niter_max[env], nmax) : nmax;
        if (P.ncon_out) P.ncon_out[env] = ncon;
        if (P.nefc_out) P.nefc_out[env] = nefc;
        if (P.warm_choice) P.warm_choice[env] = choice;
        if (P.sens_valid) P.sens_valid[env] = sens_ok;
      }
      __syncwarp();
    }
    if (lockstep) {
      group += gridDim.x;
      __syncthreads();
    } else if (P.work_counter) {
      int e = 0;
      if (lane == 0) e = atomicAdd(P.work_counter, 1);
      env = __shfl_sync(FULL_MASK, e, 0);
    } else {
      env += gridDim.x * W;
    }
  }
  if (timing)
    for (int k = 0; k < 8; k++) atomicAdd(P.stage_cycles + k, tstage[k]);
#undef STAGE_SYNC
#undef TIMED_BARRIER
}

// Geom poses of every env at its current qpos (kinematics only), for ray
// casting: gpose[env][g][12] = world position (3), rotation matrix (9, row
// major).  One warp per env; the workspace layout is the step kernel's.
__global__ void __launch_bounds__(512) mjb_geom_pose_kernel(const __grid_constant__ StepParams P, float* gpose, int ng_max) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, W = blockDim.x >> 5;
  int* dsm = reinterpret_cast<int*>(mjb_smem) + warp * P.desc_words;
  float* ws = P.gws ? P.gws + ((size_t)blockIdx.x * W + warp) * P.ws_stride : mjb_smem + W * P.desc_words + warp * P.ws_stride;
#pragma unroll 1
  for (int env = blockIdx.x * W + warp; env < P.num_envs; env += gridDim.x * W) {
    const int* src = reinterpret_cast<const int*>(P.models + P.env_model[env]);
#pragma unroll 1
    for (int k = lane; k < MJB_DESC_COPY_WORDS; k += 32) dsm[k] = __ldg(src + k);
    Env& E = *reinterpret_cast<Env*>(dsm + MJB_DESC_COPY_WORDS);
    if (lane == 0) {
      E.it = P.itab;
      E.ft = P.ftab;
      E.ws = ws;
      E.env = env;
      E.status = 0;
      E.md = reinterpret_cast<const DevModelDesc*>(dsm);
    }
    __syncwarp();
    const DevModelDesc& m = *E.md;
    const int qadr = P.env_qadr[env];
#pragma unroll 1
    for (int i = lane; i < m.nq; i += 32) ws[m.w_qpos + i] = P.qpos[qadr + i];
    __syncwarp();
    d_kinematics(E);
    float* out = gpose + (size_t)env * ng_max * 12;
#pragma unroll 1
    for (int k = lane; k < m.ngeom * 12; k += 32) {
      const int g = k / 12, q = k % 12;
      out[k] = q < 3 ? ws[m.w_gxpos + 3 * g + q] : ws[m.w_gxmat + 9 * g + (q - 3)];
    }
    __syncwarp();
  }
}

namespace {

// The dynamic shared-memory limit of a kernel is a function attribute of the
// current device.  Every launch and occupancy query goes through this helper,
// which only ever raises the attribute and remembers, per device and kernel,
// the largest value set so far; a sim created later with a smaller workspace
// therefore never lowers the limit below what an earlier sim launches with.
constexpr int kAttrDevices = 64;
enum { kAttrStep = 0, kAttrStepConvex = 1, kAttrGeomPose = 2, kAttrKernels = 3 };
std::mutex g_attr_mutex;
size_t g_attr_smem[kAttrDevices][kAttrKernels];

template <class Kernel>
cudaError_t raise_smem_limit(Kernel kernel, int slot, size_t smem_bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kAttrDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_attr_mutex);
  if (smem_bytes <= g_attr_smem[dev][slot]) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
  if (e == cudaSuccess) g_attr_smem[dev][slot] = smem_bytes;
  return e;
}

}  // namespace

cudaError_t mjb_launch_geom_pose(const StepParams& P, float* gpose, int ng_max, int warps_per_block, size_t smem_bytes, cudaStream_t stream) {
  cudaError_t e = raise_smem_limit(mjb_geom_pose_kernel, kAttrGeomPose, smem_bytes);
  if (e != cudaSuccess) return e;
  int grid = (P.num_envs + warps_per_block - 1) / warps_per_block;
  if (P.gws && grid > P.gws_blocks) grid = P.gws_blocks;   // one HBM workspace per resident warp
  mjb_geom_pose_kernel<<<grid, warps_per_block * 32, smem_bytes, stream>>>(P, gpose, ng_max);
  return cudaGetLastError();
}

// P.convex selects the instance with the GJK / EPA collider (models with
// general convex pairs); both instances share every other stage.
cudaError_t mjb_launch_step(const StepParams& P, int grid, int warps_per_block, size_t smem_bytes, cudaStream_t stream) {
  cudaError_t e = P.convex ? raise_smem_limit(mjb_step_kernel<true>, kAttrStepConvex, smem_bytes)
                           : raise_smem_limit(mjb_step_kernel<false>, kAttrStep, smem_bytes);
  if (e != cudaSuccess) return e;
  if (P.convex) mjb_step_kernel<true><<<grid, warps_per_block * 32, smem_bytes, stream>>>(P);
  else mjb_step_kernel<false><<<grid, warps_per_block * 32, smem_bytes, stream>>>(P);
  return cudaGetLastError();
}

cudaError_t mjb_occupancy(int warps_per_block, size_t smem_bytes, int convex, int* blocks_per_sm) {
  if (convex) {
    cudaError_t e = raise_smem_limit(mjb_step_kernel<true>, kAttrStepConvex, smem_bytes);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, mjb_step_kernel<true>, warps_per_block * 32, smem_bytes);
  }
  cudaError_t e = raise_smem_limit(mjb_step_kernel<false>, kAttrStep, smem_bytes);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, mjb_step_kernel<false>, warps_per_block * 32, smem_bytes);
}
