// Launch parameters of the fused physics-step kernel (POD, host and device).
#pragma once
#include <stdint.h>

#include "devmodel.h"

struct StepParams {
  // model tables
  const DevModelDesc* models;
  const int* itab;
  const float* ftab;

  // batch layout: per-env model id and offsets into the state arrays
  int num_envs;
  const int* env_model;
  const int* env_qadr;   // into qpos
  const int* env_vadr;   // into qvel / qacc_warm / qacc_pred
  const int* env_uadr;   // into ctrl / rand_gain
  const int* env_badr;   // into body-indexed outputs and rand_mass

  // state (env-major records, HBM-resident)
  float* qpos;
  float* qvel;
  const float* ctrl;
  float* qacc_warm;
  const float* qacc_pred;   // predicted warm start (nullable)

  int convex;               // 1: some model has a general convex pair or an elliptic cone (kernel instance with GJK / EPA and the cone solver)
  int nsub;                 // substeps per launch (same ctrl)
  int max_iter;             // <= 0: model default
  int* work_counter;        // persistent scheduling queue head (nullable = static env mapping)
  int lockstep;             // 1: the warps of a CTA run each stage together (barrier between stages)
  unsigned long long* stage_cycles;  // nullable: per-stage SM clock totals (lockstep mode, 8 stages)
  int ws_stride;            // floats of workspace per warp
  float* gws;               // non-null: workspaces in HBM (ws_stride floats per resident warp, by global warp index)
                            // for models whose workspace exceeds shared memory; shared memory then holds the descriptors only
  int gws_blocks;           // CTAs the HBM workspaces cover
  int desc_words;           // 32-bit words of each warp's shared-memory slot: the DevModelDesc copy, then the env context
  int itab_smem;            // words of the model int table (itab) copied into shared memory after the workspaces, read by
                            // every stage in place of itab; 0: the stages read itab from global memory

  // per-env statistics of this launch
  int* status;
  int* niter_sum;
  int* niter_max;
  int* ncon_out;
  int* nefc_out;
  int* warm_choice;

  // values recorded on the last substep (nullable)
  float* rec_xpos;
  float* rec_xquat;
  float* rec_scom;
  float* rec_cinert;
  float* rec_cvel;
  float* rec_qfrc_actuator;
  float* rec_cfrc_ext;
  float* rec_qacc;

  // sensors of the last substep's start state (nullable): sensordata at
  // env_sadr[env]; accelerometers keep the previous substep's frame linear
  // velocity (3 floats per accelerometer at env_aadr[env]) and a per-env
  // flag saying it is valid
  float* sensordata;
  const int* env_sadr;
  float* sens_prev;
  const int* env_aadr;
  int* sens_valid;

  // parity/debug outputs on the last substep (nullable)
  float* dbg_contacts;      // [B][dbg_ncon_max][MJB_CONTACT_FLOATS]
  int dbg_ncon_max;
  float* dbg_efc;           // [B][dbg_nefc_max][4]: type, force, D, aref
  int dbg_nefc_max;
  float* dbg_vec;           // [B][4*dbg_nv_max]: qacc_smooth, qfrc_smooth, qacc, qfrc_constraint
  int dbg_nv_max;

  // per-env randomisation (nullable)
  const float* rand_mass;      // [badr + body]
  const float* rand_friction;  // [env]
  const float* rand_gain;      // [uadr + actuator]
  const float* rand_com;       // [3 badr + 3 body + k]: COM offset in the body frame
  const float* rand_drag;      // [env_fadr + free joint]: quadratic drag coefficient
  const int* env_fadr;

  // learned warm start: feature rows written after each substep (nullable):
  // qpos[feat_qskip:nq], qvel, converged qacc, then MJB_FEAT_CONTACTS x
  // (contact normal, distance) in contact order, zero padded
  // feat_body = 1 (models made only of free bodies, children of the world):
  // one row per body instead, [B][nbody - 1][feat_stride], of MJB_FEAT_BODY
  // floats: height, orientation quaternion, the body's 6 velocities and 6
  // converged accelerations, then its first MJB_FEAT_BODY_CONTACTS contacts
  // in contact order as (normal along the force on this body, distance,
  // contact point minus body position), zero padded
  float* features;             // [B][feat_stride]
  int feat_stride;
  int feat_qskip;
  int feat_body;
  // fused learned warm start (per-env models, lockstep CTAs of 4, 8 or 16
  // warps; nn_w[0] null = off): after the constraint build of every substep
  // the CTA evaluates a 4-layer GELU MLP on the feature rows of its envs
  // (qpos[feat_qskip:], qvel, qacc_smooth, previous qacc, ctrl, first
  // MJB_FEAT_CONTACTS contacts as normal and distance; nn_in_raw values) and
  // offers qacc_prev + out_mean + out_std * y to the Newton solver.  Weights
  // are bf16 [nn_rows][nn_cols] per layer (K contiguous), biases fp32.
  const uint16_t* nn_w[4];
  const float* nn_b[4];
  int nn_rows[4], nn_cols[4];
  const float* nn_in_mean;
  const float* nn_in_istd;
  const float* nn_out_mean;
  const float* nn_out_std;
  int nn_in_raw;
  int nn_nout;
  // training pairs of the fused warm start written by the kernel (nullable):
  // row s * num_envs + env holds the nn_in_raw features of substep s (taken
  // after its constraint build) and the converged qacc minus the previous
  // one (nv floats); single-model batches
  float* pair_x;
  float* pair_t;
  float* nn_pred_out;          // debug capture (nullable): the fused prediction of the last substep, at env_vadr
  float* nn_feat_out;          // debug capture (nullable): the fused input features of the last substep, [B][nn_in_raw]
  int stats_accumulate;        // 1: add this launch's Newton iterations to niter_sum / max into niter_max
  int poison_workspace;        // 1: fill each env's shared workspace with NaN before its first stage (test aid)
};

#define MJB_FEAT_CONTACTS 16
#define MJB_FEAT_BODY_CONTACTS 4
#define MJB_FEAT_BODY (17 + 7 * MJB_FEAT_BODY_CONTACTS)
