// Device-side model descriptor shared by host and kernels.
//
// Every model constant the step needs lives in two flat HBM tables (ints and
// floats) that stay L2-resident; a POD descriptor per model holds sizes and
// offsets into them plus the per-env shared-memory workspace layout.  This
// replaces the reference's string-baked GLSL constants (forward.hpp:84-106,
// collision.hpp:505-515) so one kernel serves any model, and several models in
// one launch.
#pragma once

#define MJB_CONTACT_FLOATS 16  // pos3 frame9 dist pair(bits) dim includemargin

// per-warp shared-memory slot of the step kernels: the model descriptor copy
// (MJB_DESC_COPY_WORDS 32-bit words), then the warp's env context
// (MJB_ENV_SLOT_WORDS words)
#define MJB_DESC_COPY_WORDS ((int)(sizeof(DevModelDesc) / 4))
#define MJB_ENV_SLOT_WORDS 16

// alignas(16): the per-warp shared-memory copies of the descriptor precede
// the workspaces, which need 16-byte alignment for vector loads
struct alignas(16) DevModelDesc {
  // sizes
  int nq, nv, nu, nbody, njnt, ngeom, npair, nlimit, nfloss, nlevel, nmesh;
  int ncon_max, nefc_max;
  int cone, disableflags, iterations, ls_iterations, implicit;
  float timestep, gravity[3], tolerance, impratio, scale;  // scale = 1/(meaninertia*max(1,nv))

  // int table offsets
  int i_body_parentid, i_body_rootid, i_body_jntadr, i_body_jntnum, i_body_dofadr, i_body_dofnum, i_body_subtreesize;
  int i_level_start, i_level_body, i_child_start, i_child_list;
  int i_jnt_type, i_jnt_qposadr, i_jnt_dofadr;
  int i_dof_bodyid, i_dof_jntid, i_dof_parentid;
  int i_geom_type, i_geom_bodyid, i_geom_dataid;
  int i_pair;    // 6 per pair: g1 g2 b1 b2 condim maxcon
  int i_limit;   // 3 per limited joint: jnt dof qposadr
  int i_floss;   // 1 per frictionloss dof: dof
  int neq, i_eq;  // joint / tendon equalities: 5 ints each (kind 0 joint 1 tendon, obj1, obj2 or -1, qposadr1, qposadr2);
                  // obj = dof for joints, tendon id for tendons
  int i_act;     // 7 per actuator: dof qposadr gaintype biastype ctrllimited forcelimited tendon (-1 = joint transmission)
  int ntendon, i_ten, i_wrap;  // tendons: 3 ints each (wrapadr wrapnum limited); 3 per wrap element: type (1 joint, 2 pulley,
                               // 3 site, 4 sphere, 5 cylinder) then (dof, qposadr) / (0, 0) / (site, body) / (geom, side site or -1)
  int i_site_body;             // body of each site
  int ntfloss, i_tfloss;       // tendons with frictionloss (tendon ids)
  int ntlimit, i_tlimit;       // limited tendons (tendon ids)
  int npten, i_pten;           // tendons with stiffness or damping (tendon ids)
  int ngcomp, i_gcomp;   // bodies with gravity compensation (body ids)
  int nfree, i_free;     // free joints in MJCF order (dof address of each)
  int nsensor, nsensordata, nsens_acc;
  int i_sensor;  // MJB_SENSOR_INTS per sensor: mjtSensor type (-1 = reads zero), adr, dim, body, root body, a, b, accelerometer slot
  int i_mesh;    // 2 per mesh: vertadr vertnum

  // float table offsets
  int f_body_pos, f_body_quat, f_body_ipos, f_body_iquat, f_body_mass, f_body_inertia;
  int f_jnt_pos, f_jnt_axis, f_jnt_stiffness, f_qpos0, f_qpos_spring;
  int f_dof_armature, f_dof_damping, f_dof_damping_implicit, f_dof_invweight0;
  int f_geom_pos, f_geom_quat, f_geom_size, f_geom_rbound;
  int f_pair;    // 16 per pair: margin includemargin friction(5) solref(2) solimp(5) invw_t invw_r
  int f_limit;   // 10 per limit: lo hi margin solref(2) solimp(5)
  int f_floss;   // 8 per frictionloss dof: floss solref(2) solimp(5)
  int f_eq;      // 15 per joint equality: qpos0 ref1, ref2, polycoef(5), solref(2), solimp(5), invweight
  int f_act;     // 11 per actuator: gear gain(3) bias(3) ctrlrange(2) forcerange(2)
  int f_wrap;    // 1 per wrap: joint coef or pulley divisor
  int f_site;    // 3 per site: position in its body
  int f_ten;     // MJB_TEN_FLOATS per tendon (layout below)
  int f_sensor;  // MJB_SENSOR_FLOATS per sensor: object frame in its body (pos 3, quat 4), actuator gear
  int f_gcomp;   // gravcomp per body
  float magnetic[3];
  int f_mesh_vert;

  // per-env shared-memory workspace (float offsets from the warp's base)
  int ws_size;
  int w_qpos, w_qvel, w_ctrl, w_x, w_xwarm;
  int w_scom, w_cdof, w_M, w_qfs, w_qas, w_qfa, w_vec;   // w_vec: 8*nv solver vectors
  int w_ten;     // per tendon [length, velocity, J(nv)] of the current substep
  int w_tseg;    // kinematics-region scratch: straight pieces of one spatial tendon path (9 floats each)
  int w_con, w_rowcon;
  // phase region K (kinematics / dynamics), aliased by region S (solver)
  int w_xpos, w_xquat, w_xmat, w_xipos, w_xanchor, w_xaxis, w_gxpos, w_gxmat, w_cinert, w_crb, w_cvel, w_cdofdot, w_cacc, w_tmp;
  int w_J, w_efc, w_H, w_active, w_nz;   // w_nz: max(nv, 8) ints: nonzero columns of one row (row-sparse H build,
                                         // nv > 64), or the Newton inverse mode's row-set words (nv <= 32)
  int ldh;       // leading dimension of H / its factor at w_H: nv rounded up to 4 for nv <= 32 (then 32 floats of
                 // 16-byte aligned column scratch follow the nv x ldh matrix), nv otherwise
};

// per-tendon floats: range lo, hi, margin, frictionloss, stiffness, damping,
// lengthspring lo, hi, solref_lim(2), solimp_lim(5), solref_fri(2),
// solimp_fri(5), invweight0, length0
#define MJB_TEN_FLOATS 24
enum { TEN_LO = 0, TEN_HI, TEN_MARGIN, TEN_FLOSS, TEN_STIFF, TEN_DAMP, TEN_SPRLO, TEN_SPRHI, TEN_SRLIM, TEN_SILIM = 10, TEN_SRFRI = 15,
       TEN_SIFRI = 17, TEN_INVW = 22, TEN_LEN0 = 23 };

#define MJB_SENSOR_INTS 8
#define MJB_SENSOR_FLOATS 8

// efc row metadata stride (floats) in the workspace: aref D floss type y
// force q con; models with elliptic cones carry three more fields per row
// for the Newton Hessian: HD (the row's diagonal weight: D in its quadratic
// zone, else 0; for a cone's friction rows in the middle zone the tangent
// curvature), HA (the rank-1 cone term's coefficient) and HU (the
// tangent-projection term's coefficient)
#define MJB_EFC_FIELDS 8
#define MJB_EFC_FIELDS_ELLIPTIC 11
enum { EFC_AREF = 0, EFC_D, EFC_FLOSS, EFC_TYPE, EFC_Y, EFC_FORCE, EFC_Q, EFC_CON, EFC_HD, EFC_HA, EFC_HU };
// ROW_ELLIPTIC: an elliptic contact's normal row (floss = mu_0 / sqrt(impratio));
// ROW_ELLFRIC: its friction rows, which follow it (floss = that direction's mu)
enum { ROW_FRICTION = 0, ROW_LIMIT = 1, ROW_PYRAMID = 2, ROW_FRICTIONLESS = 3, ROW_ELLIPTIC = 4, ROW_EQUALITY = 5, ROW_ELLFRIC = 6 };

// status bits (per env, OR over substeps)
enum {
  MJB_STATUS_BADSTATE = 1,
  MJB_STATUS_BADQACC = 2,
  MJB_STATUS_CONTACT_OVERFLOW = 4,
  MJB_STATUS_EFC_OVERFLOW = 8,
  MJB_STATUS_UNSUPPORTED_PAIR = 16,
};
